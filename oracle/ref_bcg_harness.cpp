/*
 * ref_bcg_harness.cpp -- runs the reference's own decoder (bcg.cuh, compiled
 * for the host through ref_shim.h) over a loaded graph.  TEST INFRASTRUCTURE
 * ONLY: the Makefile in this directory compiles it twice, once against
 * GT/src/bcg.cuh (-DREF_TREE_GT) and once against LE/src/bcg.cuh, into
 * oracle/_ref/libref_bcg_{gt,le}.so.  Nothing from the reference is copied;
 * the header is included from where it lies.
 *
 * Entry points (C ABI, plain pointers):
 *   ref_decode_offset(offset_words, n, ubl, lens_out)
 *       the reference's decode_offset kernel body (bcg.cuh decode_offset),
 *       executed once per emulated thread: lens_out[u] = length field u.
 *   ref_degree(words, offsets, v)          BCGVertex(v, ...).outd
 *   ref_get_vertex(words, offsets, v, i)   BCGVertex(v, ...).get_vertex(i)
 *   ref_decode_all(words, offsets, n, rowptr, cols)
 *       get_vertex(i) for every (v, i), written as CSR.
 */
#include "ref_shim.h"
#include "bcg.cuh"

extern "C" {

void ref_decode_offset(uint32_t *offset_words, uint64_t n, uint32_t ubl, uint64_t *lens_out) {
  const unsigned threads = 256;
  blockDim.x = threads;
  gridDim.x = 1;
  blockIdx.x = 0;
  for (unsigned t = 0; t < threads; t++) {
    threadIdx.x = t;
    decode_offset(offset_words, (Offset_t *)lens_out, (VertexID_t)n, (uint8_t)ubl);
  }
}

int64_t ref_degree(const uint32_t *words, const uint64_t *offsets, int32_t v) {
  BCGVertex bv(v, words, offsets[v]);
  return bv.outd;
}

int64_t ref_get_vertex(const uint32_t *words, const uint64_t *offsets, int32_t v, int32_t i) {
  BCGVertex bv(v, words, offsets[v]);
  return bv.get_vertex(i);
}

int ref_decode_all(const uint32_t *words, const uint64_t *offsets, uint64_t n,
                   uint64_t *rowptr, uint32_t *cols) {
  uint64_t acc = 0;
  for (uint64_t v = 0; v < n; v++) {
    rowptr[v] = acc;
    BCGVertex bv((VertexID_t)v, words, offsets[v]);
    acc += (uint64_t)bv.outd;
  }
  rowptr[n] = acc;
  if (!cols) return 0;
  for (uint64_t v = 0; v < n; v++) {
    BCGVertex bv((VertexID_t)v, words, offsets[v]);
    for (int32_t i = 0; i < bv.outd; i++) cols[rowptr[v] + i] = (uint32_t)bv.get_vertex(i);
  }
  return 0;
}

}  // extern "C"
