// Host shim that compiles the reference's own CPU checks — validate() and
// report() from validate.h:34-127 — unmodified, from the reference source
// tree (include path given by oracle/Makefile). TEST INFRASTRUCTURE ONLY:
// used to pin the oracle against the reference's own invariants and
// edge-count convention. The reference's comm.h guards its CUDA globals
// behind COMM_HEADER / EXTERN (comm.h:30-182); defining both skips them, and
// the three items validate.h needs from comm.h are supplied here with the
// reference's values (depth_t = unsigned char, INFTY = 0xFF, comm.h:69,131).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#define COMM_HEADER
#define EXTERN
#define INFTY ((unsigned char)0xff)
static int g_validate_times = 1;
#define VALIDATE_TIMES g_validate_times

#include "validate.h"

extern "C" {

// Runs the reference validate() `times` random reached vertices deep.
// depth: uint8 per vertex (0xFF = unreached), beg/csr: int32 like the
// reference's in-memory graph (graph.hpp:60-88).
int ref_validate(const uint8_t* depth, const int32_t* beg, const int32_t* csr, int32_t V, int32_t times) {
  g_validate_times = times;
  return validate<int, int, unsigned char>(const_cast<unsigned char*>(depth), const_cast<int*>(beg),
                                           const_cast<int*>(csr), V);
}

void ref_report(const int32_t* beg, const uint8_t* depth, int32_t V, int32_t* tr_edges, int32_t* tr_verts) {
  int e = 0, v = 0;
  report<int, int, unsigned char>(e, v, const_cast<int*>(beg), const_cast<unsigned char*>(depth), V);
  *tr_edges = e;
  *tr_verts = v;
}

}  // extern "C"
