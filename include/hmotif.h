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

/* Files in the reference programs' formats.
 *   HM_FMT_ESCHER: space-separated vertex ids >= 1 per line, '#' comments
 *     (dynamicHyperGraph/utils/utils.cpp:88-130 loadHypergraphFromFile; vertex
 *     v is node v - 1);
 *   HM_FMT_MOCHY: comma-separated node ids >= 0 per line
 *     (MoCHy-master/read_data.cpp:8-45; repeated ids in a line count once);
 *   HM_FMT_THYME: "n1,n2,...<TAB>time" (THyMe-main/code/read_data.cpp:22-57;
 *     times must be integers).
 * A graph read from a file has n_nodes = largest node id + 1. */
#define HM_FMT_ESCHER 0
#define HM_FMT_MOCHY 1
#define HM_FMT_THYME 2
int hm_hostgraph_read(const char* path, int format, hm_hostgraph** out);
int hm_hostgraph_write(const hm_hostgraph* hg, const char* path, int format);
int hm_hostgraph_from_csr(const uint64_t* offsets, const uint32_t* members, uint32_t n_edges, uint32_t n_nodes,
                          const int64_t* times, hm_hostgraph** out);

/* ---- contexts --------------------------------------------------------- */
typedef struct hm_ctx hm_ctx;
typedef struct hm_graph hm_graph;

/* A context binds one CUDA device and one stream; every device byte the
 * engine allocates through it is charged against mem_budget_bytes (0 = the
 * device's free memory at creation). Calls on one context are serialised.
 * Replaces the per-store cudaMalloc bookkeeping of CBSTOperations
 * (dynamicHyperGraph/structure/operations.cu:359-374), which exits the
 * process on any CUDA error. */
int hm_ctx_create(int device, size_t mem_budget_bytes, hm_ctx** out);
int hm_ctx_destroy(hm_ctx* ctx);
int hm_ctx_memory(const hm_ctx* ctx, size_t* used_bytes, size_t* budget_bytes);
/* The context's cudaStream_t, as void* so this header needs no CUDA types. */
void* hm_ctx_stream(const hm_ctx* ctx);
/* Test hook: after n further successful device allocations, allocations fail
 * with HM_ERR_NOMEM (n < 0 switches the hook off). */
int hm_debug_fail_allocations_after(long long n);
/* Walk order of the touched-triple counts on graph g: 0 = each neighbour's
 * higher-(degree, id) neighbours (the default, rebuilt after each batch),
 * 1 = its higher-id neighbours, read straight from the id-sorted rows (what
 * pooled server stores use). Counts are the same either way; tests run both. */
int hm_debug_touch_orientation(hm_graph* g, int by_id);
/* Walk of the static count on graph g: 1 (the default) walks oriented rows
 * grouped by the member each neighbour shares with the row owner, and counts
 * the triangles of a pair sharing one member u through the neighbours that
 * share only u by the group's size counts instead of visiting them; 0 visits
 * every oriented entry. Counts are the same either way; tests run both. */
int hm_debug_static_groups(hm_graph* g, int on);

/* ---- the device store ------------------------------------------------- */
/* Builds H2V (hyperedge -> sorted members), V2H (node -> sorted hyperedges)
 * and H2H (hyperedge -> adjacent hyperedges with overlap sizes) on the
 * device from a host CSR: hyperedge e (id e) has members
 * members[offsets[e] .. offsets[e+1]), node ids < n_nodes. timestamps may be
 * NULL (static graph) or hold one int64 per hyperedge (temporal graph).
 * Replaces constructCBST (dynamicHyperGraph/structure/operations.cu:31-80)
 * for all three stores plus the host H2H builder hyperedgeAdjacency
 * (dynamicHyperGraph/utils/utils.cpp:399-427). */
int hm_graph_build(hm_ctx* ctx, const uint64_t* offsets, const uint32_t* members, uint32_t n_edges,
                   uint32_t n_nodes, const int64_t* timestamps, hm_graph** out);
int hm_graph_destroy(hm_graph* g);

typedef struct hm_graph_info_t {
  uint32_t n_slots;     /* ids in use or free: 0 .. n_slots-1 */
  uint32_t n_live;
  uint32_t n_nodes;
  int32_t temporal;
  uint64_t n_members;   /* H2V entries */
  uint64_t n_adjacent;  /* H2H entries (both directions) */
  uint64_t n_oriented;  /* oriented H2H entries (0 until the first count) */
  uint64_t device_bytes;/* bytes charged to the context */
} hm_graph_info_t;
int hm_graph_info(const hm_graph* g, hm_graph_info_t* info);

/* Member lists of live hyperedges ids[0..n): offsets_out[0..n] (CSR) and
 * members_out (capacity members_cap). Replaces findAndPrint / findContents
 * (dynamicHyperGraph/structure/operations.cu:425-433, kernel/find.cu:26-51),
 * which only print. HM_ERR_NOT_LIVE if an id is free or out of range. */
int hm_graph_query(hm_graph* g, const uint32_t* ids, uint32_t n, uint64_t* offsets_out, uint32_t* members_out,
                   size_t members_cap);

/* One update batch: delete the live hyperedges del_ids[0..n_del) (each at
 * most once), then insert n_ins hyperedges given as a CSR (ins_offsets has
 * n_ins + 1 entries starting at 0; members as in hm_graph_build). Inserted
 * hyperedges take the smallest free ids first, ascending (ids freed by this
 * batch included), then new ids after the largest; the ids are written to
 * assigned_ids_out (n_ins entries, may be NULL). If delta30_out is not NULL it
 * receives the exact change of the 30 static classes (new minus old), counted
 * on the device from the triples the batch touches only.
 * Replaces deleteCBST / unfillCBST / insertCBST / fillCBST
 * (dynamicHyperGraph/structure/operations.cu:82-356, 439-453) on H2V, V2H and
 * H2H together, the host rebuild of the updated graph
 * (dynamicHyperGraph/src/main.cu:333-342), and computeMotifCountsDelta
 * (dynamicHyperGraph/include/motif_update.hpp:13-19,
 * src/HMotifCountUpdate.cu:228-301), whose result is not exact in general.
 * Temporal graphs are immutable (HM_ERR_STATE). */
int hm_graph_apply_batch(hm_graph* g, const uint32_t* del_ids, uint32_t n_del, const uint64_t* ins_offsets,
                         const uint32_t* ins_members, uint32_t n_ins, uint32_t* assigned_ids_out,
                         int64_t* delta30_out);
/* hm_graph_apply_batch ordered on a caller's stream: the batch's device work
 * starts after the work already queued on `stream` (a cudaStream_t; NULL is
 * the legacy default stream), and work queued on `stream` afterwards sees the
 * updated store and, if d_delta30 (device memory, 30 int64) is not NULL, the
 * exact delta there. The host returns once the batch is sequenced: a batch
 * reads sizes back from the device between its steps, so the call does wait
 * on the context stream, but never on the caller's. HM_ERR_STATE if `stream`
 * is being captured into a CUDA graph. The reference's batch calls end in a
 * device synchronize (dynamicHyperGraph/structure/operations.cu:82-356). */
int hm_graph_apply_batch_async(hm_graph* g, const uint32_t* del_ids, uint32_t n_del, const uint64_t* ins_offsets,
                               const uint32_t* ins_members, uint32_t n_ins, uint32_t* assigned_ids_out,
                               int64_t* d_delta30, void* stream);

/* Keyed fill: live hyperedge ids[i] gains the node ids
 * values[prefix[i-1] .. prefix[i]) (prefix[-1] = 0; prefix holds the inclusive
 * end of each id's values, the reference's insertPrefixSizes) and keeps its
 * id. Members are a set: values it already holds are ignored. If delta30_out
 * is not NULL it receives the exact change of the 30 static classes. Each id
 * at most once per call; HM_ERR_NOT_LIVE if one is not live (nothing
 * changes). Replaces fillCBST / CBSTOperations::insert(insertKeys,
 * insertPayload, insertPrefixSizes) on H2V (dynamicHyperGraph/include/
 * structure.hpp:38,54; structure/operations.cu:82-127, 417-419), with V2H
 * and H2H kept in step. */
int hm_graph_fill(hm_graph* g, const uint32_t* ids, uint32_t n, const uint32_t* values, const uint64_t* prefix,
                  int64_t* delta30_out);
/* Keyed unfill: the same with the values removed from each hyperedge's
 * members (values it does not hold are ignored); a hyperedge left with no
 * members stays live, with no neighbours. Replaces unfillCBST
 * (dynamicHyperGraph/structure/operations.cu:439-453, kernel/unfill.cu:4-52). */
int hm_graph_unfill(hm_graph* g, const uint32_t* ids, uint32_t n, const uint32_t* values, const uint64_t* prefix,
                    int64_t* delta30_out);

/* The ids of the live hyperedges in ascending order; *n_out receives their
 * number (out may be NULL to query it). */
int hm_graph_live_ids(const hm_graph* g, uint32_t* out, uint32_t cap, uint32_t* n_out);

/* ---- counts ------------------------------------------------------------ */
/* 30-class counts of the connected triples that contain at least one of the
 * live hyperedges ids[0..n) (repeats ignored). The exact recount of a batch
 * is this count for the inserted ids after it minus this count for the
 * deleted ids before it. */
int hm_count_touching30(hm_graph* g, const uint32_t* ids, uint32_t n, uint64_t out30[HM_N_STATIC_CLASSES]);

/* MoCHy's 26 static h-motif counts over all connected hyperedge triples.
 * Replaces computeMotifCounts (dynamicHyperGraph/include/motif.hpp:10-13,
 * src/HMotifCount.cu:97-125), which returns nothing and counts closed
 * triangles only; the numbers are those of MoCHy main_exact
 * (MoCHy-master/main_exact.cpp:91-137). */
int hm_count_static(hm_graph* g, uint64_t out26[HM_N_STATIC_MOTIFS]);
/* The same in the reference's 30-bin order (classes 0, 1, 4, 6 are non-zero
 * only when hyperedges repeat). */
int hm_count_static30(hm_graph* g, uint64_t out30[HM_N_STATIC_CLASSES]);

/* The same counts as hm_count_touching30, for callers that cannot allocate
 * device memory while they run (a serving thread that must not block on the
 * allocator or fail for want of memory mid-request, code held to a fixed
 * memory reservation). No counterpart in the reference. d_ids (n ids) and
 * d_out30 (30 uint64) are device buffers owned by the caller; stream is a
 * cudaStream_t, and NULL is CUDA's legacy default stream (torch's default
 * stream): the kernels run on it after the work already queued there, and
 * after any work the engine left on the context stream. All scratch lives in one 8 MiB
 * device array that the library sets aside when it is loaded: graphs of at
 * most 2^21 hyperedge slots, at most 2^20 distinct ids per call. The first
 * call on a device looks the array up and configures the kernels; make it
 * before any stream capture. Calls share the array, so calls that overlap on
 * the GPU race: serialise them. Returns when the counts are written;
 * HM_ERR_NOT_LIVE if an id is not a live hyperedge (the others are counted). */
int hm_count_touching30_noalloc(hm_graph* g, const uint32_t* d_ids, uint32_t n, uint64_t* d_out30, void* stream);

/* THyMe's 96 temporal h-motif counts of a temporal graph (built with
 * timestamps) for the window delta: every event a and the connected triples
 * of the projection of the events with t_a - delta <= t <= t_a that contain
 * it, repeated node-sets collapsed into one hyperedge with several
 * occurrences (THyMe-main/code/main_thymeP.cpp:155-368). Events with equal
 * timestamps are processed in input order; the order of two occurrences is
 * decided by a strict comparison of their times, as THyMe compares them
 * (main_thymeP.cpp:313-323), a tie counting as "c before b" with b the
 * hyperedge of the pair whose node-set comes first in the input (THyMe's own
 * numbering, which its input shuffle randomises). HM_ERR_LIMIT if an event
 * has more than 4096 distinct neighbours inside its window. There is no temporal counter of
 * these 96 motifs in the reference's GPU code (its 3-layer strict-increasing
 * kernel, temporalDynamicHMotif/src/temporal_count.cu:91-217, bins 30 classes
 * of a different definition). */
int hm_count_temporal(hm_graph* g, int64_t delta, uint64_t out96[HM_N_TEMPORAL_MOTIFS]);
/* The same, asynchronous: queued after the work already on `stream` (a
 * cudaStream_t; NULL is the legacy default stream), the 96 counts land in
 * d_out96 (device memory) and work queued on `stream` afterwards sees them;
 * the call returns without waiting (the first count of a graph builds its
 * time-ordered index first and waits for that). If an event has more than
 * 4096 distinct neighbours inside its window, all 96 counts read 2^64 - 1
 * (the synchronous call returns HM_ERR_LIMIT). HM_ERR_STATE if `stream` or
 * the context stream is being captured into a CUDA graph. The reference's
 * counters are host programs with no stream (THyMe-main/code/
 * main_thymeP.cpp:117-388). */
int hm_count_temporal_async(hm_graph* g, int64_t delta, uint64_t* d_out96, void* stream);

/* Partial 30-class counts over one shard of the centres: the sum over
 * shard = 0 .. n_shards-1 equals hm_count_static30. One shard per GPU, each
 * GPU holding a replica of the graph, gives the multi-GPU count with a
 * single 30 x uint64 sum across ranks. */
int hm_count_static30_shard(hm_graph* g, uint32_t shard, uint32_t n_shards, uint64_t out30[HM_N_STATIC_CLASSES]);

/* The 30-class static count, asynchronous: queued after the work already on
 * `stream` (a cudaStream_t; NULL is CUDA's legacy default stream, which is
 * also torch's default stream; pass hm_ctx_stream(ctx) for the context
 * stream), it writes the counts to d_out30 (device memory, 30 uint64) and
 * returns without waiting; work queued on `stream` afterwards sees them. The
 * first call on a graph (and the first after an update) prepares the
 * oriented rows and the work list and waits for that. Do not change the graph
 * or count it again until the stream has passed the count. HM_ERR_STATE if
 * `stream` or the context stream is being captured into a CUDA graph. After
 * this call hm_graph_timings reports the static phase times as -1 (not
 * measured). The reference's calls all end in a device synchronize
 * (dynamicHyperGraph/src/HMotifCount.cu:97-125). */
int hm_count_static30_async(hm_graph* g, uint64_t* d_out30, void* stream);

/* Algorithmic bytes of one static count of this graph (for rooflines):
 * b_static follows the reference-equivalent merge algorithm
 * (MoCHy-master/main_exact.cpp:91-129): store read once
 * (4 nnz(H2V) + 8 nnz(H2H)), sum over id-ordered adjacent pairs of
 * 8 (d+(a) + d+(b)) with d+ the neighbours of larger id, and
 * 4 (|a| + |b|) per pair that closes a triangle. kernel_bytes is what this
 * engine's kernels read. Runs one extra diagnostic count (slow). */
typedef struct hm_traffic_t {
  uint64_t store_bytes;
  uint64_t merge_bytes;
  uint64_t closed_pair_bytes;
  uint64_t b_static;
  uint64_t probes;          /* hash probes of the closed phase */
  uint64_t kernel_bytes;
  uint64_t closed_triangles;
} hm_traffic_t;
int hm_graph_traffic(hm_graph* g, hm_traffic_t* t);

/* ---- launch schedules, and their autotuner --------------------------------
 * Static count: the closed-triangle phase runs three persistent launch
 * shapes over one heaviest-first list of centres, split by the length d of
 * each centre's oriented row: d <= warp_row one warp per centre
 * (warp_row <= 128), d <= small_row one 256-thread block per centre with a
 * 4096-slot table (warp_row <= small_row <= 2048), longer rows blocks with an
 * 8192-slot table. Touched-triple count (the delta of every update batch):
 * the same three shapes per marked hyperedge m by the length of its row:
 * <= touch_warp_row one warp (<= 128), <= touch_mid_row 4096-slot blocks
 * (touch_warp_row <= touch_mid_row <= 2048), longer rows 1024-thread blocks
 * with a 16384-slot table or a global table. Counts never depend on the
 * schedule; speed does. Default {128, 2048, 128, 2048}. The reference has
 * one launch shape, a thread per hyperedge
 * (dynamicHyperGraph/src/HMotifCount.cu:97-125,
 * src/HMotifCountUpdate.cu:150-226). */
typedef struct hm_schedule {
  uint32_t warp_row;
  uint32_t small_row;
  uint32_t touch_warp_row;
  uint32_t touch_mid_row;
} hm_schedule;
int hm_graph_set_schedule(hm_graph* g, const hm_schedule* s);
int hm_graph_get_schedule(const hm_graph* g, hm_schedule* s);

#define HM_TUNE_MAX_CANDIDATES 16
typedef struct hm_tune_report {
  /* static count: (warp_row, small_row) candidates, [0] the default */
  uint32_t n_candidates;
  uint32_t best;          /* index of the pair now in use */
  uint32_t sample_stride; /* every sample_stride-th centre of the work list was timed */
  uint32_t sampled;       /* centres in the timed sample */
  uint32_t rows[HM_TUNE_MAX_CANDIDATES][2];
  float ms[HM_TUNE_MAX_CANDIDATES];       /* closed-phase device time of the sample */
  /* touched-triple count: (touch_warp_row, touch_mid_row) candidates */
  uint32_t touch_n_candidates;
  uint32_t touch_best;
  uint32_t touch_sampled; /* live hyperedges marked in the timed count */
  uint32_t touch_rows[HM_TUNE_MAX_CANDIDATES][2];
  float touch_ms[HM_TUNE_MAX_CANDIDATES]; /* wall time of the count of the sample */
  float tune_ms;          /* wall time of the whole tuning call */
} hm_tune_report;
/* Times each candidate schedule of the two counts with the same input for
 * all candidates, and keeps the fastest of each; a default stays unless
 * another is at least 2 % faster. Static count: the closed phase on a
 * strided sample of the centres (sample_stride 0: at most 65536 centres,
 * 1: all), CUDA-event time; the candidates vary warp_row only (small_row
 * 2048), as a sparse sample misjudges which rows share N+ in L2.
 * Touched-triple count: the count of every n-th live hyperedge (about 4096
 * of them, as a deletion batch marks them).
 * report may be NULL. */
int hm_graph_autotune(hm_graph* g, uint32_t sample_stride, hm_tune_report* report);

/* Device times of the last count / update call on this graph (CUDA events
 * on the context stream). */
typedef struct hm_timings_t {
  float open_ms;     /* open-pair phase of the static count */
  float closed_ms;   /* closed-triangle phase of the static count */
  float count_ms;    /* whole static count */
  float update_ms;   /* last batch update */
  float temporal_ms; /* last temporal count */
  uint64_t closed_triangles;
} hm_timings_t;
int hm_graph_timings(const hm_graph* g, hm_timings_t* t);

/* Algorithmic bytes of the last temporal count (for rooflines). For each
 * event a, N(a) is the set of distinct hyperedges of its delta-window
 * projection that share a node with it, d(a) = |N(a)|, and d_a(b) the degree
 * of b in that projection. The bytes follow the reference algorithm's walk
 * (THyMe-main/code/main_thymeP.cpp:219-334: the neighbours of a, then the
 * neighbours of each of them), 8 bytes per adjacency entry:
 *   b_temp = sum_a 8 d(a) + 8 sum_{b in N(a)} d_a(b),
 * with sum_{b in N(a)} d_a(b) = d(a) + 2 closed_pairs(a) + open_pairs(a)
 * (pairs of neighbours of a that overlap; pairs (b, c) with c adjacent to b
 * but not to a). Zero before the first temporal count. */
typedef struct hm_temporal_traffic_t {
  uint64_t events;
  int64_t delta;
  uint64_t window_neighbours; /* sum_a d(a) */
  uint64_t closed_pairs;      /* sum_a closed_pairs(a) */
  uint64_t open_pairs;        /* sum_a open_pairs(a) */
  uint64_t b_temp;
} hm_temporal_traffic_t;
int hm_graph_temporal_traffic(const hm_graph* g, hm_temporal_traffic_t* t);

/* Class of a 7-bit region pattern: static class 0..29 or temporal motif
 * 0..95 (-1 if the pattern is not a connected triple). Bits: exclusive parts
 * of x, y, z; x&y only; y&z only; z&x only; x&y&z. */
int hm_classify_static(int pattern);
int hm_classify_temporal(int pattern);

/* The reference's vertex-triad counts (temporalDynamicHMotif/src/type1.cu,
 * type2.cu, type3.cu and their host versions type{1,2,3}.cpp):
 *   out3[0] type 1: sum over hyperedges of C(|e|, 3);
 *   out3[1] type 2: sum over adjacent pairs i < j with a = |i & j| >= 2 and
 *           both |i| - a, |j| - a > 0 of C(a, 2) (|i| - a) (|j| - a);
 *   out3[2] type 3: sum over pairwise-adjacent triples of x y z, x, y, z the
 *           pairwise overlaps minus the triple overlap, all three > 0. */
int hm_count_vertex_triads(hm_graph* g, uint64_t out3[3]);

/* ---- Three-layer temporal window, strictly increasing count --------------
 * Replaces TemporalCBSTOperations / TemporalHypergraphIndex, a 3-slot ring of
 * stores (temporalDynamicHMotif/include/temporal_structure.hpp:22-80,
 * include/temporal_adjacency.hpp:9-19), and computeTemporalMotifCountsStrictInc
 * (include/temporal_count.hpp:10-16, src/temporal_count.cu:91-217): closed
 * triples (i of Older, j of Middle, k of Newest) with layer-local ids
 * i < j < k and all pairwise overlaps non-empty, by the 30 static classes,
 * without the reference's cap of 1024 candidates per middle hyperedge.
 * Hyperedge ids are 0-based per layer; node ids < n_nodes. */
typedef struct hm_window hm_window;
#define HM_LAYER_OLDER 0
#define HM_LAYER_MIDDLE 1
#define HM_LAYER_NEWEST 2
int hm_window_create(hm_ctx* ctx, uint32_t n_nodes, hm_window** out);
int hm_window_destroy(hm_window* w);
/* construct(layer, ...): the layer's hyperedges, replacing what it held */
int hm_window_set_layer(hm_window* w, int layer, const uint64_t* offsets, const uint32_t* members, uint32_t n_edges);
/* rotate(): Middle becomes Older, Newest Middle, Older Newest (contents kept) */
int hm_window_rotate(hm_window* w);
/* resetLayer(layer): the layer becomes empty */
int hm_window_reset_layer(hm_window* w, int layer);
/* fill / unfill (fillCBST / unfillCBST): add or remove vertices of existing
 * hyperedges; prefix[i] is the inclusive end of ids[i]'s values */
int hm_window_fill(hm_window* w, int layer, const uint32_t* ids, uint32_t n, const uint32_t* values,
                   const uint64_t* prefix);
int hm_window_unfill(hm_window* w, int layer, const uint32_t* ids, uint32_t n, const uint32_t* values,
                     const uint64_t* prefix);
/* applyTemporalDeltasFromFile: lines "A <hyperedge> v..." / "R <hyperedge> v..."
 * (1-based ids and vertices) on the Newest layer; removals applied first */
int hm_window_apply_deltas_file(hm_window* w, const char* path);
int hm_window_layer_size(const hm_window* w, int layer, uint32_t* n_edges);
int hm_window_count30(hm_window* w, uint64_t out30[HM_N_STATIC_CLASSES]);

/* ---- Serving: many resident graphs behind one request loop ---------------
 * No reference counterpart: the reference drivers call applyIncrementalUpdates
 * + computeMotifCountsDelta (dynamicHyperGraph/src/main.cu:232-244,
 * src/HMotifCountUpdate.cu:228-301) and computeMotifCounts
 * (src/HMotifCount.cu:97-125) once per request, which is what
 * HM_SERVE_PER_REQUEST does here.
 *
 * A server owns a set of graphs, each with its own hyperedge ids (0-based,
 * smallest free id first, exactly as hm_graph_apply_batch assigns them) and
 * its own node ids. Requests (an update batch with its exact delta, or a full
 * count) are queued; a loop thread serves them in arrival order per graph.
 *   HM_SERVE_BATCHED: all graphs live node-disjoint in one pooled store;
 *     each round the loop admits the oldest waiting request of every graph
 *     that fits the limits and the memory budget, and serves them all with
 *     one sequence of launches (the deleted-side count, one store update, one
 *     touched-triple count that also counts the queried graphs), splitting
 *     the counters per request. Requests that arrive meanwhile join the next
 *     round.
 *   HM_SERVE_PER_REQUEST: one store per graph, one hm_graph_apply_batch /
 *     hm_count_static30 call per request, in arrival order.
 * Both give identical results for the same requests. */
typedef struct hm_server hm_server;

#define HM_SERVE_BATCHED 0
#define HM_SERVE_PER_REQUEST 1

typedef struct hm_serve_config {
  int32_t mode;                /* HM_SERVE_BATCHED or HM_SERVE_PER_REQUEST */
  uint32_t max_batch_requests; /* requests per round, 0 = no limit */
  uint64_t max_batch_edits;    /* deletions + insertions per round, 0 = no limit */
  size_t mem_budget_bytes;     /* admission budget, 0 = the context's budget */
  /* 1: once a count request has counted a graph in full, the server keeps
   * that graph's counts current by adding the exact delta of each of its
   * updates, and answers its later count requests from them with no device
   * work; 0: every count request counts its graph in full. The counts are
   * the same either way. */
  int32_t count_from_deltas;
  int32_t pad_;
} hm_serve_config;

#define HM_REQ_UPDATE 0
#define HM_REQ_COUNT 1

typedef struct hm_serve_result {
  uint64_t ticket;
  uint32_t graph;
  int32_t kind;                             /* HM_REQ_UPDATE or HM_REQ_COUNT */
  int32_t status;                           /* HM_OK or the request's own error */
  uint32_t n_assigned;                      /* update: ids given to its insertions */
  int64_t delta30[HM_N_STATIC_CLASSES];     /* update: exact change of the counts */
  uint64_t counts30[HM_N_STATIC_CLASSES];   /* count: the graph's counts */
  double submit_ms, start_ms, done_ms;      /* server clock (ms since creation) */
  uint32_t round_requests;                  /* requests served in its round */
  uint32_t pad_;
} hm_serve_result;

typedef struct hm_serve_stats_t {
  uint64_t rounds;
  uint64_t requests_done;
  uint64_t requests_failed;
  uint64_t edits_done;
  uint64_t waiting;          /* queued, not yet served */
  uint64_t deferred_budget;  /* admissions deferred by the memory budget */
  double busy_ms;            /* loop time spent serving rounds */
  size_t device_bytes;       /* the context's device memory in use */
} hm_serve_stats_t;

int hm_serve_create(hm_ctx* ctx, const hm_serve_config* cfg, hm_server** out);
/* Adds a graph (before hm_serve_start); its id is written to graph_out. */
int hm_serve_add_graph(hm_server* s, const uint64_t* offsets, const uint32_t* members, uint32_t n_edges,
                       uint32_t n_nodes, uint32_t* graph_out);
/* Builds the device stores and starts the loop thread. */
int hm_serve_start(hm_server* s);
/* Queue requests; inputs are copied. Validation errors of a request are
 * reported in its result, and leave its graph unchanged. */
int hm_serve_submit_update(hm_server* s, uint32_t graph, const uint32_t* del_ids, uint32_t n_del,
                           const uint64_t* ins_offsets, const uint32_t* ins_members, uint32_t n_ins,
                           uint64_t* ticket_out);
int hm_serve_submit_count(hm_server* s, uint32_t graph, uint64_t* ticket_out);
/* Blocks until the request is served; hands its result over once. assigned
 * (may be NULL) receives the insertions' ids, up to cap. */
int hm_serve_wait(hm_server* s, uint64_t ticket, hm_serve_result* out, uint32_t* assigned, uint32_t cap);
/* Blocks until every queued request has been served. */
int hm_serve_drain(hm_server* s);
int hm_serve_stats(hm_server* s, hm_serve_stats_t* out);
/* Current live ids of one graph (ascending); call when drained. */
int hm_serve_live_ids(hm_server* s, uint32_t graph, uint32_t* out, uint32_t cap, uint32_t* n_out);
/* Stops the loop (after serving what is queued) and frees the stores. */
int hm_serve_destroy(hm_server* s);

#ifdef __cplusplus
}
#endif

#endif /* HMOTIF_H */
