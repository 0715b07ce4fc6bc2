/*
 * hm_oracle.c - CPU restatement of the reference's exact h-motif counters.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA engine:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it, and never as the thing measured or shipped. The engine has no CPU
 * path and never calls into this file.
 *
 * It restates, in plain C with sorted arrays in place of hash maps:
 *   - MoCHy exact (MoCHy-master/main_exact.cpp:47-129): the 30 static classes
 *     over all connected hyperedge triples (open ones at their centre, closed
 *     ones once at the smallest id), reported as 26 motifs;
 *   - THyMe+ exact (THyMe-main/code/main_thymeP.cpp:155-368): the 96 temporal
 *     h-motifs over a sliding delta window, with repeated node-sets collapsed
 *     into one static hyperedge carrying a list of timestamps;
 *   - two brute-force definition oracles (all triples / all event triples)
 *     for tiny inputs, used to cross-check the two restatements.
 *
 * Parity pin: tests compare these functions with outputs of the reference's
 * own programs (MoCHy main_exact / main_exact_par, THyMe main_thyme /
 * main_thymeP, compiled from the reference sources into oracle/_ref by
 * oracle/build_ref.sh) stored as fixtures under tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "hm_oracle.h"

/* ------------------------------------------------------------------------ */
/* Classification of one triple from its seven Venn regions.                 */
/* ------------------------------------------------------------------------ */

/*
 * Static class (0..29, -1 if the triple is not connected). The reference
 * tabulates this as a 128-entry array (MoCHy-master/motif_id.cpp:5-22,
 * dynamicHyperGraph/kernel/motif_utils.cuh:6-23). Here it is derived from
 * the structure of the pattern: with p = number of non-empty pairwise-only
 * regions,
 *   g>0, p=0: 1 + #exclusive regions                      -> 1..4
 *   g>0, p=1: pair (u,w) + loner z, by (excl u + excl w, excl z) -> 5..10
 *   g>0, p=2: hub h (in both pair regions) + two ends, by (excl h, #excl ends) -> 11..16
 *   g>0, p=3: 17 + #exclusive                             -> 17..20
 *   g=0, p=2: as g>0, p=2, from 21                        -> 21..26
 *   g=0, p=3: 27 + #exclusive                             -> 27..30
 * and the result is that 1-based number minus one.
 */
int hmo_static_class_bits(int pattern) {
  const int ea = pattern & 1, eb = (pattern >> 1) & 1, ec = (pattern >> 2) & 1;
  const int pab = (pattern >> 3) & 1, pbc = (pattern >> 4) & 1, pca = (pattern >> 5) & 1;
  const int g = (pattern >> 6) & 1;
  const int p = pab + pbc + pca, nex = ea + eb + ec;
  static const int pair_rank[2][3] = {{0, 1, 3}, {2, 4, 5}}; /* [excl loner][excl pair members] */
  int one_based = 0;
  if (p == 3) {
    one_based = (g ? 17 : 27) + nex;
  } else if (p == 2) {
    int hub_ex = pca && pab ? ea : (pab && pbc ? eb : ec);
    int ends_ex = nex - hub_ex;
    one_based = (g ? 11 : 21) + hub_ex + 2 * ends_ex;
  } else if (g && p == 1) {
    int loner_ex = pab ? ec : (pbc ? ea : eb);
    one_based = 5 + pair_rank[loner_ex][nex - loner_ex];
  } else if (g && p == 0) {
    one_based = 1 + nex;
  }
  return one_based - 1;
}

static int region_pattern(int sa, int sb, int sc, int cab, int cbc, int cca, int g) {
  int a = sa - (cab + cca) + g, b = sb - (cbc + cab) + g, c = sc - (cca + cbc) + g;
  int d = cab - g, e = cbc - g, f = cca - g;
  return (a > 0) | ((b > 0) << 1) | ((c > 0) << 2) | ((d > 0) << 3) | ((e > 0) << 4) | ((f > 0) << 5) |
         ((g > 0) << 6);
}

int hmo_static_class(int sa, int sb, int sc, int cab, int cbc, int cca, int g) {
  return hmo_static_class_bits(region_pattern(sa, sb, sc, cab, cbc, cca, g));
}

/*
 * THyMe's temporal numbering (THyMe-main/code/motif_id.cpp:25-42) is a
 * bijection between the 96 connected region patterns, written with the three
 * hyperedges in time order (1st, 2nd, 3rd), and motif numbers 1..96. It has
 * no closed form, so it is kept as data: entry m-1 is the pattern of motif m,
 * bits (excl 1st, excl 2nd, excl 3rd, 1st&2nd, 2nd&3rd, 3rd&1st, all three).
 */
static const uint8_t kTemporalMotifPattern[96] = {
    67,  69,  70,  71,  73,  74,  82,  84,  97,  100, 75,  86,  101, 77,  78,  83,  85,  99,  102, 79,
    87,  103, 88,  104, 112, 90,  105, 116, 89,  92,  106, 108, 113, 114, 91,  94,  107, 109, 117, 118,
    93,  110, 115, 95,  111, 119, 120, 121, 122, 124, 123, 125, 126, 127, 24,  40,  48,  26,  41,  52,
    25,  28,  42,  44,  49,  50,  27,  30,  43,  45,  53,  54,  29,  46,  51,  31,  47,  55,  56,  57,
    58,  60,  59,  61,  62,  63,  65,  66,  68,  72,  80,  96,  76,  81,  98,  64};

static int g_temporal_of_pattern[128];
static int g_temporal_ready = 0;

static void temporal_init(void) {
  if (g_temporal_ready) return;
  for (int i = 0; i < 128; ++i) g_temporal_of_pattern[i] = -1;
  for (int m = 0; m < 96; ++m) g_temporal_of_pattern[kTemporalMotifPattern[m]] = m;
  g_temporal_ready = 1;
}

int hmo_temporal_class_bits(int pattern) {
  temporal_init();
  return g_temporal_of_pattern[pattern & 127];
}

/* Temporal class (0..95) of hyperedges x1, x2, x3 listed in time order. */
int hmo_temporal_class(int s1, int s2, int s3, int c12, int c23, int c31, int g) {
  return hmo_temporal_class_bits(region_pattern(s1, s2, s3, c12, c23, c31, g));
}

/* ------------------------------------------------------------------------ */
/* Small helpers over sorted uint32 lists.                                   */
/* ------------------------------------------------------------------------ */

static int cmp_u32(const void* x, const void* y) {
  uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
  return a < b ? -1 : a > b;
}

static uint32_t inter_count(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb) {
  uint32_t i = 0, j = 0, c = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j]) ++i;
    else if (a[i] > b[j]) ++j;
    else { ++c; ++i; ++j; }
  }
  return c;
}

static uint32_t inter3_count(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, const uint32_t* c,
                             uint32_t nc) {
  uint32_t i = 0, j = 0, k = 0, n = 0;
  while (i < na && j < nb && k < nc) {
    uint32_t m = a[i];
    if (b[j] > m) m = b[j];
    if (c[k] > m) m = c[k];
    if (a[i] == m && b[j] == m && c[k] == m) { ++n; ++i; ++j; ++k; continue; }
    if (a[i] < m) ++i;
    if (b[j] < m) ++j;
    if (c[k] < m) ++k;
  }
  return n;
}

/* Hyperedge lists: sorted, repeats inside one hyperedge dropped (MoCHy's
 * reader drops them, MoCHy-master/read_data.cpp:32-37). */
typedef struct {
  uint32_t n;
  uint64_t* off;
  uint32_t* mem;
} csr_t;

static void csr_free(csr_t* g) {
  free(g->off);
  free(g->mem);
  g->off = NULL;
  g->mem = NULL;
}

static int csr_from_input(uint32_t n, const uint64_t* off, const uint32_t* mem, csr_t* out) {
  out->n = n;
  out->off = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n + 1));
  out->mem = (uint32_t*)malloc(sizeof(uint32_t) * (off[n] ? off[n] : 1));
  if (!out->off || !out->mem) return -1;
  uint64_t w = 0;
  out->off[0] = 0;
  for (uint32_t e = 0; e < n; ++e) {
    uint64_t b = w;
    memcpy(out->mem + b, mem + off[e], sizeof(uint32_t) * (off[e + 1] - off[e]));
    uint64_t len = off[e + 1] - off[e];
    qsort(out->mem + b, len, sizeof(uint32_t), cmp_u32);
    for (uint64_t i = 0; i < len; ++i)
      if (i == 0 || out->mem[b + i] != out->mem[b + i - 1]) out->mem[w++] = out->mem[b + i];
    out->off[e + 1] = w;
  }
  return 0;
}

/* Projected graph: per hyperedge a, neighbours sorted by id and overlaps. */
typedef struct {
  uint64_t* off;
  uint32_t* nbr;
  uint32_t* ovl;
} adj_t;

static void adj_free(adj_t* a) {
  free(a->off);
  free(a->nbr);
  free(a->ovl);
}

/* Builds node->hyperedge lists and the projection, the way MoCHy does
 * (MoCHy-master/main_exact.cpp:56-68): walk every member's hyperedge list
 * and count how often each other hyperedge is met. */
static int build_projection(const csr_t* h, uint32_t n_nodes, adj_t* adj) {
  uint64_t nnz = h->off[h->n];
  uint64_t* voff = (uint64_t*)calloc((size_t)n_nodes + 1, sizeof(uint64_t));
  uint32_t* vlist = (uint32_t*)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
  uint64_t* cur = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n_nodes + 1));
  int64_t* seen = (int64_t*)malloc(sizeof(int64_t) * (h->n ? h->n : 1));
  uint32_t* cnt = (uint32_t*)calloc(h->n ? h->n : 1, sizeof(uint32_t));
  if (!voff || !vlist || !cur || !seen || !cnt) return -1;
  for (uint64_t i = 0; i < nnz; ++i) voff[h->mem[i] + 1]++;
  for (uint32_t v = 0; v < n_nodes; ++v) voff[v + 1] += voff[v];
  memcpy(cur, voff, sizeof(uint64_t) * ((size_t)n_nodes + 1));
  for (uint32_t e = 0; e < h->n; ++e)
    for (uint64_t i = h->off[e]; i < h->off[e + 1]; ++i) vlist[cur[h->mem[i]]++] = e;
  /* first pass: degrees */
  adj->off = (uint64_t*)calloc((size_t)h->n + 1, sizeof(uint64_t));
  if (!adj->off) return -1;
  for (uint32_t e = 0; e < h->n; ++e) seen[e] = -1;
  for (uint32_t a = 0; a < h->n; ++a) {
    uint64_t d = 0;
    for (uint64_t i = h->off[a]; i < h->off[a + 1]; ++i) {
      uint32_t v = h->mem[i];
      for (uint64_t j = voff[v]; j < voff[v + 1]; ++j) {
        uint32_t b = vlist[j];
        if (b != a && seen[b] != (int64_t)a) { seen[b] = a; ++d; }
      }
    }
    adj->off[a + 1] = adj->off[a] + d;
  }
  uint64_t total = adj->off[h->n];
  adj->nbr = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
  adj->ovl = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
  if (!adj->nbr || !adj->ovl) return -1;
  for (uint32_t e = 0; e < h->n; ++e) seen[e] = -1;
  for (uint32_t a = 0; a < h->n; ++a) {
    uint64_t w = adj->off[a];
    for (uint64_t i = h->off[a]; i < h->off[a + 1]; ++i) {
      uint32_t v = h->mem[i];
      for (uint64_t j = voff[v]; j < voff[v + 1]; ++j) {
        uint32_t b = vlist[j];
        if (b == a) continue;
        if (seen[b] != (int64_t)a) { seen[b] = a; cnt[b] = 0; adj->nbr[w++] = b; }
        cnt[b]++;
      }
    }
    uint64_t b0 = adj->off[a], len = w - b0;
    qsort(adj->nbr + b0, len, sizeof(uint32_t), cmp_u32);
    for (uint64_t k = b0; k < w; ++k) adj->ovl[k] = cnt[adj->nbr[k]];
  }
  free(voff);
  free(vlist);
  free(cur);
  free(seen);
  free(cnt);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* MoCHy exact restated (MoCHy-master/main_exact.cpp:91-129).                 */
/* ------------------------------------------------------------------------ */
/* Counts the triples owned by centres a = shard (mod n_shards): open triples
 * at their centre, closed ones at a = min, the owner rule main_exact_par
 * splits its parallel counting loop over a by (main_exact_par.cpp:122-173). The shards
 * of one n_shards partition all triples. */
int hmo_static30_shard(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint32_t n_nodes,
                       uint32_t shard, uint32_t n_shards, uint64_t out30[30]) {
  csr_t h;
  adj_t adj;
  memset(out30, 0, sizeof(uint64_t) * 30);
  if (csr_from_input(n_edges, offsets, members, &h)) return -1;
  for (uint64_t i = 0; i < h.off[n_edges]; ++i)
    if (h.mem[i] >= n_nodes) { csr_free(&h); return -2; }
  if (build_projection(&h, n_nodes, &adj)) { csr_free(&h); return -1; }
  uint32_t* inter = (uint32_t*)malloc(sizeof(uint32_t) * (HMO_MAX_EDGE + 1));
  /* Dense stand-in for MoCHy's per-hyperedge hash map of overlaps
   * (hyperedge_inter, main_exact.cpp:70-78): N(b) is scattered once per
   * (a, b) and looked up in O(1) for every c. */
  uint32_t* mk_ovl = (uint32_t*)malloc(sizeof(uint32_t) * (n_edges ? n_edges : 1));
  uint64_t* mk_tag = (uint64_t*)malloc(sizeof(uint64_t) * (n_edges ? n_edges : 1));
  for (uint32_t e = 0; e < n_edges; ++e) mk_tag[e] = UINT64_MAX;
  for (uint32_t a = 0; a < n_edges; ++a) {
    if (a % n_shards != shard) continue;
    const uint32_t* ma = h.mem + h.off[a];
    uint32_t sa = (uint32_t)(h.off[a + 1] - h.off[a]);
    for (uint64_t i = adj.off[a]; i < adj.off[a + 1]; ++i) {
      uint32_t b = adj.nbr[i], cab = adj.ovl[i];
      const uint32_t* mb = h.mem + h.off[b];
      uint32_t sb = (uint32_t)(h.off[b + 1] - h.off[b]);
      /* I_ab, materialised once per (a, b) as MoCHy does (:105-106) */
      uint32_t ni = 0, p = 0, q = 0;
      while (p < sa && q < sb) {
        if (ma[p] < mb[q]) ++p;
        else if (ma[p] > mb[q]) ++q;
        else { inter[ni++] = ma[p]; ++p; ++q; }
      }
      if (i + 1 < adj.off[a + 1])
        for (uint64_t k = adj.off[b]; k < adj.off[b + 1]; ++k) {
          mk_tag[adj.nbr[k]] = i;
          mk_ovl[adj.nbr[k]] = adj.ovl[k];
        }
      for (uint64_t j = i + 1; j < adj.off[a + 1]; ++j) {
        uint32_t c = adj.nbr[j], cca = adj.ovl[j];
        const uint32_t* mc = h.mem + h.off[c];
        uint32_t sc = (uint32_t)(h.off[c + 1] - h.off[c]);
        uint32_t cbc = mk_tag[c] == i ? mk_ovl[c] : 0;
        if (cbc) {
          if (a < b) { /* closed: counted once, at a = min (neighbours sorted, so b < c) */
            uint32_t g = inter_count(inter, ni, mc, sc);
            int k = hmo_static_class((int)sa, (int)sb, (int)sc, (int)cab, (int)cbc, (int)cca, (int)g);
            if (k >= 0) out30[k]++;
          }
        } else { /* open: counted at its centre a */
          int k = hmo_static_class((int)sa, (int)sb, (int)sc, (int)cab, 0, (int)cca, 0);
          if (k >= 0) out30[k]++;
        }
      }
    }
  }
  free(inter);
  free(mk_ovl);
  free(mk_tag);
  adj_free(&adj);
  csr_free(&h);
  return 0;
}

int hmo_static30(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint32_t n_nodes,
                 uint64_t out30[30]) {
  return hmo_static30_shard(n_edges, offsets, members, n_nodes, 0, 1, out30);
}

/* Strictly increasing three-layer count, restating the reference's
 * temporalStrictIncAdjKernel (temporalDynamicHMotif/src/temporal_count.cu:
 * 91-170): closed triples (i of the older layer, j of the middle, k of the
 * newest) with layer-local ids i < j < k and all three pairwise overlaps
 * non-empty, by static class of (|i|, |j|, |k|, C_ij, C_jk, C_ik, g). The
 * reference stops collecting candidates at 1024 per middle hyperedge; this
 * restatement has no such cap. Brute force over all (i, j, k). */
int hmo_strictinc30(const uint64_t* off0, const uint32_t* mem0, uint32_t n0, const uint64_t* off1,
                    const uint32_t* mem1, uint32_t n1, const uint64_t* off2, const uint32_t* mem2, uint32_t n2,
                    uint64_t out30[30]) {
  csr_t L0, L1, L2;
  memset(out30, 0, sizeof(uint64_t) * 30);
  if (csr_from_input(n0, off0, mem0, &L0)) return -1;
  if (csr_from_input(n1, off1, mem1, &L1)) { csr_free(&L0); return -1; }
  if (csr_from_input(n2, off2, mem2, &L2)) { csr_free(&L0); csr_free(&L1); return -1; }
  for (uint32_t j = 0; j < n1; ++j) {
    const uint32_t* mj = L1.mem + L1.off[j];
    const uint32_t sj = (uint32_t)(L1.off[j + 1] - L1.off[j]);
    for (uint32_t i = 0; i < n0 && i < j; ++i) {
      const uint32_t* mi = L0.mem + L0.off[i];
      const uint32_t si = (uint32_t)(L0.off[i + 1] - L0.off[i]);
      const uint32_t cij = inter_count(mi, si, mj, sj);
      if (!cij) continue;
      for (uint32_t k = j + 1; k < n2; ++k) {
        const uint32_t* mk = L2.mem + L2.off[k];
        const uint32_t sk = (uint32_t)(L2.off[k + 1] - L2.off[k]);
        const uint32_t cjk = inter_count(mj, sj, mk, sk);
        if (!cjk) continue;
        const uint32_t cik = inter_count(mi, si, mk, sk);
        if (!cik) continue;
        const uint32_t g = inter3_count(mi, si, mj, sj, mk, sk);
        int c = hmo_static_class((int)si, (int)sj, (int)sk, (int)cij, (int)cjk, (int)cik, (int)g);
        if (c >= 0) out30[c]++;
      }
    }
  }
  csr_free(&L0);
  csr_free(&L1);
  csr_free(&L2);
  return 0;
}

/* Vertex-triad counts of the reference's type1/type2/type3 programs
 * (temporalDynamicHMotif/src/type1.cpp:6-15, type2.cpp:17-44,
 * type3.cpp:58-94), restated over the deduplicated member lists:
 *   type1 = sum over hyperedges of C(|e|, 3);
 *   type2 = sum over adjacent pairs i < j with a = |i & j| >= 2,
 *           b = |i| - a > 0, c = |j| - a > 0 of C(a, 2) * b * c;
 *   type3 = sum over pairwise-adjacent i < j < k of x * y * z, x, y, z the
 *           pairwise overlaps minus the triple overlap, all three > 0. */
int hmo_vertex_triads(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint64_t out3[3]) {
  csr_t h;
  out3[0] = out3[1] = out3[2] = 0;
  if (csr_from_input(n_edges, offsets, members, &h)) return -1;
  for (uint32_t i = 0; i < n_edges; ++i) {
    const uint64_t si = h.off[i + 1] - h.off[i];
    if (si >= 3) out3[0] += si * (si - 1) * (si - 2) / 6;
    for (uint32_t j = i + 1; j < n_edges; ++j) {
      const uint32_t sj = (uint32_t)(h.off[j + 1] - h.off[j]);
      const uint32_t a = inter_count(h.mem + h.off[i], (uint32_t)si, h.mem + h.off[j], sj);
      if (!a) continue;
      if (a >= 2 && si > a && sj > a) out3[1] += (uint64_t)a * (a - 1) / 2 * (si - a) * (sj - a);
      for (uint32_t k = j + 1; k < n_edges; ++k) {
        const uint32_t sk = (uint32_t)(h.off[k + 1] - h.off[k]);
        const uint32_t b = inter_count(h.mem + h.off[j], sj, h.mem + h.off[k], sk);
        if (!b) continue;
        const uint32_t c = inter_count(h.mem + h.off[i], (uint32_t)si, h.mem + h.off[k], sk);
        if (!c) continue;
        const uint32_t g = inter3_count(h.mem + h.off[i], (uint32_t)si, h.mem + h.off[j], sj, h.mem + h.off[k], sk);
        if (a > g && b > g && c > g) out3[2] += (uint64_t)(a - g) * (b - g) * (c - g);
      }
    }
  }
  csr_free(&h);
  return 0;
}

/* The 26 reported motifs: classes other than 0, 1, 4, 6
 * (MoCHy-master/main_exact.cpp:133-137). */
void hmo_static26_from30(const uint64_t in30[30], uint64_t out26[26]) {
  int m = 0;
  for (int k = 0; k < 30; ++k)
    if (k != 0 && k != 1 && k != 4 && k != 6) out26[m++] = in30[k];
}

/* Brute force over all triples, for small inputs (definition check). */
int hmo_static30_brute(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint64_t out30[30]) {
  csr_t h;
  memset(out30, 0, sizeof(uint64_t) * 30);
  if (csr_from_input(n_edges, offsets, members, &h)) return -1;
#define M(e) (h.mem + h.off[e])
#define S(e) ((uint32_t)(h.off[(e) + 1] - h.off[e]))
  for (uint32_t a = 0; a < n_edges; ++a)
    for (uint32_t b = a + 1; b < n_edges; ++b) {
      uint32_t cab = inter_count(M(a), S(a), M(b), S(b));
      for (uint32_t c = b + 1; c < n_edges; ++c) {
        uint32_t cbc = inter_count(M(b), S(b), M(c), S(c));
        uint32_t cca = inter_count(M(c), S(c), M(a), S(a));
        if ((cab > 0) + (cbc > 0) + (cca > 0) < 2) continue;
        uint32_t g = inter3_count(M(a), S(a), M(b), S(b), M(c), S(c));
        int k = hmo_static_class((int)S(a), (int)S(b), (int)S(c), (int)cab, (int)cbc, (int)cca, (int)g);
        if (k >= 0) out30[k]++;
      }
    }
#undef M
#undef S
  csr_free(&h);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* THyMe+ exact restated (THyMe-main/code/main_thymeP.cpp:155-368).          */
/* ------------------------------------------------------------------------ */

typedef struct {
  const csr_t* h;
  const uint32_t* key; /* static id of each event */
} stat_ctx_t;

static int cmp_edges_ctx_h;
static const csr_t* g_sort_h;
static int cmp_edge_lex(const void* x, const void* y) {
  uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
  uint64_t la = g_sort_h->off[a + 1] - g_sort_h->off[a], lb = g_sort_h->off[b + 1] - g_sort_h->off[b];
  if (la != lb) return la < lb ? -1 : 1;
  int c = memcmp(g_sort_h->mem + g_sort_h->off[a], g_sort_h->mem + g_sort_h->off[b], la * sizeof(uint32_t));
  if (c) return c;
  return a < b ? -1 : a > b;
}

static const int64_t* g_sort_t;
static int cmp_time(const void* x, const void* y) {
  uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
  if (g_sort_t[a] != g_sort_t[b]) return g_sort_t[a] < g_sort_t[b] ? -1 : 1;
  return a < b ? -1 : a > b;
}

/* Number of pairs (x in X, y in Y) with x < y; X, Y sorted ascending
 * (main_thymeP.cpp:313-323). */
static uint64_t ordered_pairs(const int64_t* X, uint32_t nx, const int64_t* Y, uint32_t ny) {
  uint64_t n = 0;
  uint32_t j = 0;
  for (uint32_t i = 0; i < nx; ++i) {
    while (j < ny && Y[j] <= X[i]) ++j;
    n += ny - j;
  }
  return n;
}

int hmo_temporal96(uint32_t n_events, const uint64_t* offsets, const uint32_t* members, const int64_t* times,
                   int64_t delta, uint64_t out96[96]) {
  csr_t h;
  memset(out96, 0, sizeof(uint64_t) * 96);
  if (csr_from_input(n_events, offsets, members, &h)) return -1;
  if (n_events == 0) { csr_free(&h); return 0; }
  /* 1. Repeated node-sets collapse into one static hyperedge (:164-179). */
  uint32_t* byset = (uint32_t*)malloc(sizeof(uint32_t) * n_events);
  uint32_t* sid = (uint32_t*)malloc(sizeof(uint32_t) * n_events);
  uint32_t* rep = (uint32_t*)malloc(sizeof(uint32_t) * n_events); /* static id -> one event */
  for (uint32_t e = 0; e < n_events; ++e) byset[e] = e;
  g_sort_h = &h;
  qsort(byset, n_events, sizeof(uint32_t), cmp_edge_lex);
  uint32_t n_static = 0;
  for (uint32_t i = 0; i < n_events; ++i) {
    uint32_t e = byset[i];
    if (i > 0) {
      uint32_t p = byset[i - 1];
      uint64_t lp = h.off[p + 1] - h.off[p], le = h.off[e + 1] - h.off[e];
      if (!(lp == le && memcmp(h.mem + h.off[p], h.mem + h.off[e], le * sizeof(uint32_t)) == 0)) ++n_static;
    }
    sid[e] = n_static;
    rep[n_static] = e;
  }
  ++n_static;
  /* Input index of each node-set's first event: THyMe numbers node-sets in
   * the order it meets them (:164-179), which decides which of two
   * hyperedges of an instance is "b" when their occurrences tie in time. */
  uint32_t* first_in = (uint32_t*)malloc(sizeof(uint32_t) * n_static);
  for (uint32_t s = 0; s < n_static; ++s) first_in[s] = UINT32_MAX;
  for (uint32_t e = 0; e < n_events; ++e)
    if (first_in[sid[e]] == UINT32_MAX) first_in[sid[e]] = e;
  /* 2. Events in time order (:188-195), equal times by input position (THyMe
   * shuffles them, so its own counts vary between runs when times tie). */
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n_events);
  for (uint32_t e = 0; e < n_events; ++e) order[e] = e;
  g_sort_t = times;
  qsort(order, n_events, sizeof(uint32_t), cmp_time);
  /* Window state per static id: its occurrence times inside the window. */
  uint32_t* occ_n = (uint32_t*)calloc(n_static, sizeof(uint32_t));
  uint32_t* occ_first = (uint32_t*)calloc(n_static, sizeof(uint32_t)); /* index into order[] */
  int64_t* tbuf_b = (int64_t*)malloc(sizeof(int64_t) * n_events);
  int64_t* tbuf_c = (int64_t*)malloc(sizeof(int64_t) * n_events);
  uint32_t* win = (uint32_t*)malloc(sizeof(uint32_t) * n_static); /* static ids present */
  uint32_t* nbr = (uint32_t*)malloc(sizeof(uint32_t) * n_static);
  uint32_t* nbr_c = (uint32_t*)malloc(sizeof(uint32_t) * n_static);
  int64_t* mark = (int64_t*)malloc(sizeof(int64_t) * n_static);
  uint32_t* ovl_a = (uint32_t*)malloc(sizeof(uint32_t) * n_static);
  for (uint32_t s = 0; s < n_static; ++s) mark[s] = -1;
  uint32_t start = 0;
#define SM(s) (h.mem + h.off[rep[s]])
#define SS(s) ((uint32_t)(h.off[rep[s] + 1] - h.off[rep[s]]))
  for (uint32_t end = 0; end < n_events; ++end) {
    uint32_t ea = order[end], a = sid[ea];
    int64_t ta = times[ea];
    /* (1) expire events older than ta - delta (:228-234) */
    while (times[order[start]] + delta < ta) {
      uint32_t s = sid[order[start]];
      occ_n[s]--;
      ++start;
    }
    /* (2) add the new event (:237) */
    (void)occ_first;
    occ_n[a]++;
    /* static ids in the window, and occurrence times (sorted) of one id */
    uint32_t nw = 0;
    for (uint32_t k = start; k <= end; ++k) {
      uint32_t s = sid[order[k]];
      if (mark[s] != (int64_t)end) { mark[s] = end; win[nw++] = s; }
    }
    /* neighbours of a in the window projection, with overlaps */
    uint32_t na = 0, sa = SS(a);
    for (uint32_t i = 0; i < nw; ++i) {
      uint32_t s = win[i];
      ovl_a[s] = 0;
      if (s == a) continue;
      uint32_t c = inter_count(SM(a), sa, SM(s), SS(s));
      ovl_a[s] = c;
      if (c) nbr[na++] = s;
    }
    ovl_a[a] = 0;
    /* times of a static id inside the window, ascending (excluding the
     * current event when the id is a) */
#define COLLECT(sx, buf, cnt)                                               \
  do {                                                                      \
    cnt = 0;                                                                \
    for (uint32_t k = start; k < end; ++k)                                  \
      if (sid[order[k]] == (sx)) (buf)[cnt++] = times[order[k]];            \
  } while (0)
    /* (3) instances (a, b, c) and their time orderings (:243-334) */
    for (uint32_t i = 0; i < na; ++i) {
      uint32_t b = nbr[i], sb = SS(b), cab = ovl_a[b];
      /* neighbours c of b in the window */
      uint32_t nb = 0;
      for (uint32_t k = 0; k < nw; ++k) {
        uint32_t c = win[k];
        if (c == a || c == b) continue;
        if (inter_count(SM(b), sb, SM(c), SS(c))) nbr_c[nb++] = c;
      }
      uint32_t tb_n;
      COLLECT(b, tbuf_b, tb_n);
      for (uint32_t k = 0; k < nb; ++k) {
        uint32_t c = nbr_c[k], sc = SS(c), cca = ovl_a[c];
        uint32_t cbc = inter_count(SM(b), sb, SM(c), sc);
        /* closed: once per unordered {b, c}, b the node-set seen first in the input */
        if (cca && !(first_in[b] < first_in[c])) continue;
        uint32_t g = cca ? inter3_count(SM(a), sa, SM(b), sb, SM(c), sc) : 0;
        uint32_t tc_n;
        COLLECT(c, tbuf_c, tc_n);
        uint64_t bc = ordered_pairs(tbuf_b, tb_n, tbuf_c, tc_n);
        uint64_t cb = (uint64_t)tb_n * tc_n - bc;
        /* b before c before a, and c before b before a */
        int kbc = hmo_temporal_class((int)sb, (int)sc, (int)sa, (int)cbc, (int)cca, (int)cab, (int)g);
        int kcb = hmo_temporal_class((int)sc, (int)sb, (int)sa, (int)cbc, (int)cab, (int)cca, (int)g);
        if (kbc >= 0) out96[kbc] += bc;
        if (kcb >= 0) out96[kcb] += cb;
      }
      /* open at a: c adjacent to a but not to b, each unordered pair once */
      for (uint32_t j = i + 1; j < na; ++j) {
        uint32_t c = nbr[j], sc = SS(c), cca = ovl_a[c];
        if (inter_count(SM(b), sb, SM(c), sc)) continue;
        uint32_t tc_n;
        COLLECT(c, tbuf_c, tc_n);
        /* the node-set seen first in the input takes THyMe's role of b: the
         * occurrence pairs of b strictly before c go one way, the rest
         * (ties included) the other */
        uint64_t bc = first_in[b] < first_in[c] ? ordered_pairs(tbuf_b, tb_n, tbuf_c, tc_n)
                                                : (uint64_t)tb_n * tc_n - ordered_pairs(tbuf_c, tc_n, tbuf_b, tb_n);
        uint64_t cb = (uint64_t)tb_n * tc_n - bc;
        int kbc = hmo_temporal_class((int)sb, (int)sc, (int)sa, 0, (int)cca, (int)cab, 0);
        int kcb = hmo_temporal_class((int)sc, (int)sb, (int)sa, 0, (int)cab, (int)cca, 0);
        if (kbc >= 0) out96[kbc] += bc;
        if (kcb >= 0) out96[kcb] += cb;
      }
    }
    /* (4) motifs 87-95: a repeated hyperedge with one neighbour (:338-363) */
    uint32_t ta_n;
    COLLECT(a, tbuf_c, ta_n); /* earlier occurrences of a in the window */
    for (uint32_t i = 0; i < na; ++i) {
      uint32_t b = nbr[i], sb = SS(b), cab = ovl_a[b];
      uint32_t tb_n;
      COLLECT(b, tbuf_b, tb_n);
      uint64_t ab = ordered_pairs(tbuf_c, ta_n, tbuf_b, tb_n); /* old a before b */
      uint64_t ba = (uint64_t)ta_n * tb_n - ab;
      uint64_t bb = (uint64_t)tb_n * (tb_n ? tb_n - 1 : 0) / 2;
      /* (a_old, b, a) ; (b, a_old, a) ; (b_old, b, a) */
      int kab = hmo_temporal_class((int)sa, (int)sb, (int)sa, (int)cab, (int)cab, (int)sa, (int)cab);
      int kba = hmo_temporal_class((int)sb, (int)sa, (int)sa, (int)cab, (int)sa, (int)cab, (int)cab);
      int kbb = hmo_temporal_class((int)sb, (int)sb, (int)sa, (int)sb, (int)cab, (int)cab, (int)cab);
      if (kab >= 0) out96[kab] += ab;
      if (kba >= 0) out96[kba] += ba;
      if (kbb >= 0) out96[kbb] += bb;
    }
    /* (5) motif 96: three occurrences of the same node-set (:365-367) */
    if (ta_n >= 2) out96[95] += (uint64_t)ta_n * (ta_n - 1) / 2;
#undef COLLECT
  }
#undef SM
#undef SS
  free(byset); free(sid); free(rep); free(order); free(occ_n); free(occ_first); free(first_in);
  free(tbuf_b); free(tbuf_c); free(win); free(nbr); free(nbr_c); free(mark); free(ovl_a);
  csr_free(&h);
  (void)cmp_edges_ctx_h;
  return 0;
}

/* Brute force over all event triples in time order, for tiny inputs: three
 * events e1 < e2 < e3 (time order) with t3 - t1 <= delta whose node-sets form
 * a connected triple; when two or three node-sets are equal the triple counts
 * when the distinct ones overlap (THyMe's motifs 87-96). */
int hmo_temporal96_brute(uint32_t n_events, const uint64_t* offsets, const uint32_t* members, const int64_t* times,
                         int64_t delta, uint64_t out96[96]) {
  csr_t h;
  memset(out96, 0, sizeof(uint64_t) * 96);
  if (csr_from_input(n_events, offsets, members, &h)) return -1;
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n_events ? n_events : 1));
  for (uint32_t e = 0; e < n_events; ++e) order[e] = e;
  g_sort_t = times;
  qsort(order, n_events, sizeof(uint32_t), cmp_time);
#define M(e) (h.mem + h.off[e])
#define S(e) ((uint32_t)(h.off[(e) + 1] - h.off[e]))
  for (uint32_t i = 0; i < n_events; ++i)
    for (uint32_t j = i + 1; j < n_events; ++j)
      for (uint32_t k = j + 1; k < n_events; ++k) {
        uint32_t x = order[i], y = order[j], z = order[k];
        if (times[z] - times[x] > delta) continue;
        uint32_t c12 = inter_count(M(x), S(x), M(y), S(y));
        uint32_t c23 = inter_count(M(y), S(y), M(z), S(z));
        uint32_t c31 = inter_count(M(z), S(z), M(x), S(x));
        if ((c12 > 0) + (c23 > 0) + (c31 > 0) < 2) continue;
        uint32_t g = inter3_count(M(x), S(x), M(y), S(y), M(z), S(z));
        int m = hmo_temporal_class((int)S(x), (int)S(y), (int)S(z), (int)c12, (int)c23, (int)c31, (int)g);
        if (m >= 0) out96[m]++;
      }
#undef M
#undef S
  free(order);
  csr_free(&h);
  return 0;
}
