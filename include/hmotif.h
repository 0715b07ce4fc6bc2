/*
 * hmotif.h - C ABI of the B200 hypergraph motif engine.
 *
 * Every entry point returns an int status: HM_OK (0) or a negative HM_ERR_*
 * code; hm_last_error() gives the message of the calling thread's last
 * failure. Nothing in this library calls exit(). Arrays are plain host
 * pointers plus sizes; no C++ or framework types cross this boundary.
 *
 * Ids. Hyperedge ids and node ids are 0-based uint32. The reference store
 * (dynamicHyperGraph/include/structure.hpp:38-64) uses 1-based int keys with
 * 0 reserved as padding; the C++ shim in hmotif_cbst.hpp maps between the
 * two. Member lists may arrive unsorted and with repeated node ids; repeats
 * inside one hyperedge are dropped, as MoCHy's reader does
 * (MoCHy-master/read_data.cpp:32-37).
 *
 * Counts. The 26 static h-motif counts are MoCHy's "motif 1..26"
 * (MoCHy-master/main_exact.cpp:133-137): the 30 internal classes minus
 * classes 0, 1, 4 and 6, which only arise from repeated hyperedges. The 96
 * temporal counts are THyMe's motifs 1..96
 * (THyMe-main/code/main_thymeP.cpp:386-388). All counts are uint64.
 */
#ifndef HMOTIF_H
#define HMOTIF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HM_OK 0
#define HM_ERR_INVALID (-1)   /* bad argument (NULL pointer, id out of range, ...) */
#define HM_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define HM_ERR_NOMEM (-3)     /* device budget exceeded or allocation failed */
#define HM_ERR_CAPACITY (-4)  /* a caller-provided output buffer is too small */
#define HM_ERR_NOT_LIVE (-5)  /* a hyperedge id is not live */
#define HM_ERR_TIMEOUT (-6)   /* a bounded device-side wait gave up */
#define HM_ERR_STATE (-7)     /* call not valid in the object's current state */
#define HM_ERR_LIMIT (-8)     /* input beyond a documented size limit */

#define HM_N_STATIC_CLASSES 30 /* internal static classes (reference 30-bin order) */
#define HM_N_STATIC_MOTIFS 26  /* MoCHy's reported motifs */
#define HM_N_TEMPORAL_MOTIFS 96
#define HM_MAX_EDGE_SIZE 255   /* largest hyperedge (distinct members) accepted */

/* Message of the calling thread's most recent failure ("" if none). */
const char* hm_last_error(void);
/* Static description of a status code. */
const char* hm_status_string(int status);

/* ---- seeded synthetic workloads (host only) ---------------------------- */
/* Hyperedge sizes k in [k_min, k_max] with P(k) ~ k^-size_exp; members drawn
 * without replacement with P(node of popularity rank r) ~ (r + 1 + pop_offset)^-pop_exp
 * (pop_offset = 0 is plain Zipf). Members come out sorted and unique. With
 * dedupe != 0 a hyperedge equal to an earlier one is redrawn, so the result
 * holds exactly n_edges distinct hyperedges. permute_nodes != 0 maps
 * popularity ranks to node ids through a seeded permutation. */
typedef struct hm_gen_params {
  uint64_t seed;
  uint32_t n_nodes;
  uint32_t n_edges;
  uint32_t k_min;
  uint32_t k_max;
  double size_exp;
  double pop_exp;
  double pop_offset;
  int32_t dedupe;
  int32_t permute_nodes;
} hm_gen_params;

/* Bursty timestamps: bursts start as a Poisson process with rate burst_rate,
 * each holds events_per_burst events with exponential gaps of mean gap_mean;
 * the sorted times are rescaled onto [0, span] (span > 0), rounded, and made
 * strictly increasing. */
typedef struct hm_burst_params {
  double burst_rate;
  uint32_t events_per_burst;
  double gap_mean;
  int64_t span;
} hm_burst_params;

typedef struct hm_hostgraph hm_hostgraph;
typedef struct hm_hostgraph_info {
  uint32_t n_edges;
  uint32_t n_nodes;
  uint64_t n_members;
  const uint64_t* offsets; /* n_edges + 1 */
  const uint32_t* members; /* n_members */
  const int64_t* timestamps; /* n_edges, or NULL */
  uint64_t redraws;        /* duplicate hyperedges redrawn */
} hm_hostgraph_info;

int hm_gen_static(const hm_gen_params* p, hm_hostgraph** out);
int hm_gen_temporal(const hm_gen_params* p, const hm_burst_params* b, hm_hostgraph** out);
/* One update batch: round(n_edits * insert_fraction) insertions drawn from the
 * laws of p (popularity tables from p->seed, draws from batch_seed) and the
 * rest deletions drawn uniformly without replacement from live_ids, written
 * sorted to del_ids_out (capacity >= n_edits). */
int hm_gen_batch(const hm_gen_params* p, uint64_t batch_seed, const uint32_t* live_ids, uint32_t n_live,
                 uint32_t n_edits, double insert_fraction, uint32_t* del_ids_out, uint32_t* n_del_out,
                 hm_hostgraph** ins_out);
int hm_hostgraph_view(const hm_hostgraph* hg, hm_hostgraph_info* info);
void hm_hostgraph_free(hm_hostgraph* hg);

#ifdef __cplusplus
}
#endif

#endif /* HMOTIF_H */
