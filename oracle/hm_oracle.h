/*
 * hm_oracle.h - CPU restatement of the reference's exact counters.
 * TEST INFRASTRUCTURE ONLY (the checker); see hm_oracle.c.
 */
#ifndef HM_ORACLE_H
#define HM_ORACLE_H

#include <stdint.h>

#define HMO_MAX_EDGE 255

#ifdef __cplusplus
extern "C" {
#endif

int hmo_static_class_bits(int pattern);
int hmo_static_class(int sa, int sb, int sc, int cab, int cbc, int cca, int g);
int hmo_temporal_class_bits(int pattern);
int hmo_temporal_class(int s1, int s2, int s3, int c12, int c23, int c31, int g);

int hmo_static30(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint32_t n_nodes,
                 uint64_t out30[30]);
int hmo_static30_shard(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint32_t n_nodes,
                       uint32_t shard, uint32_t n_shards, uint64_t out30[30]);
int hmo_strictinc30(const uint64_t* off0, const uint32_t* mem0, uint32_t n0, const uint64_t* off1,
                    const uint32_t* mem1, uint32_t n1, const uint64_t* off2, const uint32_t* mem2, uint32_t n2,
                    uint64_t out30[30]);
int hmo_vertex_triads(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint64_t out3[3]);
void hmo_static26_from30(const uint64_t in30[30], uint64_t out26[26]);
int hmo_static30_brute(uint32_t n_edges, const uint64_t* offsets, const uint32_t* members, uint64_t out30[30]);

int hmo_temporal96(uint32_t n_events, const uint64_t* offsets, const uint32_t* members, const int64_t* times,
                   int64_t delta, uint64_t out96[96]);
int hmo_temporal96_brute(uint32_t n_events, const uint64_t* offsets, const uint32_t* members,
                         const int64_t* times, int64_t delta, uint64_t out96[96]);

#ifdef __cplusplus
}
#endif

#endif
