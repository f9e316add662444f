// Shared device-side definitions of the attract_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "attract_b200.h"

namespace att {

// Device view of one AttGrid: everything the scoring kernels read per bead.
struct __align__(16) KGrid {
  float ox, oy, oz, inv_s;        // origin, 1/spacing
  float fdx1, fdy1, fdz1;         // inner dim - 1 (float, for the range test)
  float fex1, fey1, fez1;         // outer dim2 - 1
  float ext;                      // gridextension
  float plateau, plateau2, plateau_x2;  // plateau, its square, twice it
  int dx, dy, dz;                 // inner points
  int dx2, dy2, dz2;              // outer points
  int n_types;
  int n_rec, n_rtypes, n_ltypes;
  int has_outer;
  long long type_stride;          // bricks per type (inner + outer)
  long long n_inner;              // inner bricks per type
  const float4* bricks;           // NULL: no potential grid
  const uint2* nb_hdr;            // NULL: no neighbour grid
  const uint16_t* nb_list;        // CSR entries (the records' overflow)
  const unsigned char* nb_rec;    // fixed-size records, one per inner grid point
  int nb_rec_bytes;               // record size
  int nb_inline;                  // entries held inline in a record
  float nb_scale;                 // list-grid points per inner spacing (1, 2 or 4)
  int ndy, ndz;                   // list-grid points along y and z
  long long n_list;               // CSR entries, records (= inner grid points), bricks (all types):
  long long n_vox;                //   sizes for the bounds checks of ATT_BOUNDS_CHECK builds
  long long n_bricks;
  const float4* rec;
  const float4* pair;             // [n_ltypes][n_rtypes][2] float4
};

enum Mode { MODE_EVAL = 0, MODE_EVAL_MAT = 1, MODE_MIN = 2, MODE_BWD = 3, MODE_QUAT = 4 };

struct KParams {
  KGrid grid[ATT_MAX_GRIDS];
  const float4* lig_beads;
  const int* lig_off;
  const AttSegment* segs;
  const int* seg_tile;
  int n_segs, n_tiles;
  int n_grids, n_lig, max_beads;  // bounds of the segment / conformer / bead-range checks
  int n_pose_rows;
  const float* pose_in;
  float* pose_out;
  const int* pose_lig;
  float* adam;           // [B][12] or NULL
  float* energy;         // [B]
  float* grad;           // [B][6] or [B][16]
  int* status;           // [B] or NULL
  int* counter;          // work queue (MODE_MIN), NULL = static tiles
  unsigned long long* stats;
  const float* dLdE;     // MODE_BWD
  float* dLdpose;        // MODE_BWD
  float* dgrid_inner;    // MODE_BWD
  float* dgrid_outer;    // MODE_BWD
  int steps;
  int grad_mode;
  int quirk;
  float gravity;
  float lr_rot, lr_trans, b1, b2, eps;
  int step0;
  int rec_slot;          // bytes of a neighbour-record slot in shared memory (max over grids)
  int test_flags;        // reserved (0)
  int qs_n;               // MODE_QUAT: SCHEMA stages, epochs / learning rate / gravity on-off per stage
  int qs_epochs[ATT_MAX_STAGES];
  float qs_lr[ATT_MAX_STAGES];
  int qs_grav[ATT_MAX_STAGES];
  float eps_root;
  long long n_lig_beads;   // rows of lig_beads
  long long n_dgrid_inner, n_dgrid_outer;
};

__device__ __forceinline__ float4 ldg_f4(const float4* p) { return __ldg(p); }

// Grid bricks are streamed: keep them out of L1 so that the receptor, pair
// table and ligand beads stay resident there.
__device__ __forceinline__ float4 ldg_stream_f4(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ uint2 ldg_u2(const uint2* p) { return __ldg(p); }

// One 32-byte row (two float4) in a single 256-bit read-only load: a gather
// of such rows touches each cache line once per instruction instead of twice.
// p must be 32-B aligned.
__device__ __forceinline__ void ldg_f4x2(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ unsigned ldg_u16(const uint16_t* p) {
  return (unsigned)__ldg(reinterpret_cast<const unsigned short*>(p));
}

}  // namespace att
