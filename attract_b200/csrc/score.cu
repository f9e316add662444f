// Scoring and fused minimisation kernels (K1 energrad / minimise, K2 adjoint).
//
// A pose is served by a team of S lanes (S = 8, 16 or 32: 32/S poses per warp).
// Team lane l owns ligand beads l, l+S, ... (K beads per lane, N <= K*S); the
// ligand-frame coordinates stay in registers for the whole minimisation.  One
// evaluation of a pose runs in three phases:
//
//  A  every owner lane moves its beads, computes the voxel, and -- when its
//     shared-memory slot does not already hold them -- copies the bead's
//     128-byte grid brick (the 8 trilinear corners of the voxel, (E, Fx, Fy,
//     Fz) each) and the fixed-size neighbour record of its nearest list-grid
//     point into its slots of the warp's shared memory (16-byte cp.async
//     through L2, each lane's completed by its own wait_group: in the
//     minimisers every lane copies for its own beads; the single-evaluation
//     modes spread the warp's copies over all 32 lanes and end with a warp
//     barrier).  A bead moves ~0.1 A per ADAM step against 0.9 A cells, so
//     only a few percent of a minimisation's evaluations copy anything;
//  D  each owner interpolates its brick from shared memory (rotated corner
//     order: conflict-free) and adds the grid term.  In the minimisers a
//     lane's brick copies and record copies are two cp.async groups, and
//     phase D waits only for the bricks: the records, which change more
//     often (list points are 4x finer than cells), land while it runs;
//  C  neighbour pairs: the owners write their beads' list entries into the
//     team's pair buffer, and the team's lanes take the pairs round-robin
//     (balanced whatever the per-bead list lengths).
// The adjoint (K2) runs C before D, which measured faster for its grid scatter.
//
// Energy, dE/dt and the torque are linear in every corner / pair contribution,
// so each lane accumulates its own share and the team sums 7 values with
// xor-shuffles per evaluation.  The rigid-body ADAM step runs on team lanes
// 0..5 between evaluations; a persistent launch pulls tiles of poses from a
// work counter.  No thread waits on a flag or a barrier object: a lane waits
// only for its own cp.async copies and at warp barriers.
//
// Semantics follow test5.py (sjdv1982/attract-jax):
//   transform            [x,1] @ mat                    test5.py:315-317
//   inner/outer select   0 <= v < dim-1                 test5.py:288-294
//   trilinear            floor/ceil weights             test5.py:255-266
//   grid gradient        -interpolated force            test5.py:307-311
//   list lookup          floor(v + 0.5), inner only     test5.py:322-336
//   pair term            nonbon(d^2) - E(plateau)       test5.py:186-229
//   pair gradient        custom JVP plateau correction  test5.py:220-229
//   total, gravity       E_grid + E_nb + 0.1|t|^2       test5.py:404-420
#include <math.h>

#include <type_traits>

#include "common.cuh"

namespace att {

// ---------------------------------------------------------------------------
// shared memory and copy helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// 16-byte global -> shared copy through L2 (cp.async.cg), completed by
// cp.async.wait_group in the issuing thread; both addresses 16-B aligned.
// (Measured against one bulk copy per brick or record completing on a warp
// mbarrier: 3.8 % faster in the minimiser, per lane; 11 % faster for single
// evaluations, spread over the warp.)
__device__ __forceinline__ void cp16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ void cp_commit_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's committed copy groups are pending
// (the older groups complete first)
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Loads with a fixed state space.  A list entry comes either from the
// shared-memory record or from global memory; written as two distinct
// instructions the compiler cannot fold them into one load of a selected
// address (a global-only load given a shared address is an address-space
// fault).
__device__ __forceinline__ unsigned lds_u16(const void* p) {
  unsigned short v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}

__device__ __forceinline__ unsigned lds_u32(const void* p) {
  unsigned v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}

__device__ __forceinline__ uint4 lds_u128(const void* p) {  // p 16-byte aligned
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(smem_u32(p)) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ldg_nc_u16(const uint16_t* p) {
  unsigned short v;
  asm volatile("ld.global.nc.u16 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}

// per-bead records shared by the team
struct __align__(16) BeadPos {  // moved bead; w = ligand type (int bits)
  float x, y, z;
  int lt;
};
struct __align__(16) BeadArm {  // lever arm for the torque (Q x) or ligand-frame x (dE/dmat)
  float x, y, z, pad;
};

// device-wide error word of the scoring kernels (ATT_KERR_* bits), read and
// cleared by att_kernel_status()
__device__ int g_kernel_error = 0;

// Debug builds (-DATT_BOUNDS_CHECK) check every computed index against its
// buffer before the access, skip the access when it is out of range, and
// record the first failure (check code, index, bound) for att_kernel_debug_info.
__device__ unsigned long long g_kernel_debug[3] = {0ull, 0ull, 0ull};
#ifdef ATT_BOUNDS_CHECK
__device__ __noinline__ void bounds_report(int code, long long a, long long b) {
  atomicOr(&g_kernel_error, ATT_KERR_BOUNDS);
  if (atomicCAS(&g_kernel_debug[0], 0ull, (unsigned long long)code) == 0ull) {
    g_kernel_debug[1] = (unsigned long long)a;
    g_kernel_debug[2] = (unsigned long long)b;
  }
}
#define ATT_CHECK(cond, code, a, b) ((cond) ? true : (bounds_report((code), (a), (b)), false))
#else
#define ATT_CHECK(cond, code, a, b) true
#endif

// shared memory of one warp: per bead slot a 128-B brick, a neighbour-record
// slot of rec_slot bytes, a 16-B moved-bead record and, in the modes that
// accumulate dE/dmat, a 16-B ligand-frame record; the pair buffers of the
// warp's teams (pairs_per_bead(K) u32 words per bead slot, plus S words of
// padding per team so that teams start in different banks).
// A team with more pairs than its buffer holds takes several windows; with
// several beads per lane, 4 words per slot keep a block's shared memory small
// enough for one more block per SM (13 % faster on 40-bead ligands at 2 beads
// per lane, 51 % at 4) while most teams still need a single window.
__host__ __device__ constexpr int pairs_per_bead(int K) { return K == 1 ? 8 : 4; }
__host__ __device__ inline int rec_stride(int rec_slot) { return rec_slot ? rec_slot + 16 : 0; }
__host__ __device__ inline size_t pair_buffer_bytes(int K) { return (size_t)32 * (pairs_per_bead(K) * K + 1) * 4; }
// (the bead arms are held only by the modes that accumulate dE/dmat; the
// others take the lever arm from the bead record)
__host__ __device__ inline size_t warp_smem_bytes(int K, int rec_slot, bool arms = true) {
  return (size_t)32 * K * (128 + rec_stride(rec_slot) + sizeof(BeadPos) + (arms ? sizeof(BeadArm) : 0)) +
         pair_buffer_bytes(K);
}

template <int S>
__device__ __forceinline__ float team_sum(float v) {
#pragma unroll
  for (int off = S / 2; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Sums of six values over a team of S lanes, on every lane of the team.  A
// reduce-scatter butterfly: the first three levels (lane bits S/2, S/4, S/8)
// each send half of the values still held and keep the other half (a lane
// with the level's bit clear keeps the first half), the remaining levels sum
// the one value left, so the six sums take 8 / 7 / 6 shuffles at S = 32 /
// 16 / 8 instead of 30 / 24 / 18; each sum is then broadcast from the lanes
// that hold it (team lane 0, S/4, S/8, S/2, S/2 + S/4, S/2 + S/8).  Each sum
// is formed once, so every lane receives the same bits.
template <int S>
__device__ __forceinline__ void team_sum6(float& a0, float& a1, float& a2, float& a3, float& a4, float& a5,
                                          int lane) {
  static_assert(S >= 8, "three scatter levels");
  constexpr unsigned F = 0xffffffffu;
  constexpr int H1 = S / 2, H2 = S / 4, H3 = S / 8;
  const bool h1 = lane & H1, h2 = lane & H2, h3 = lane & H3;
  float k0 = h1 ? a3 : a0, k1 = h1 ? a4 : a1, k2 = h1 ? a5 : a2;  // kept: (a0 a1 a2) or (a3 a4 a5)
  k0 += __shfl_xor_sync(F, h1 ? a0 : a3, H1);
  k1 += __shfl_xor_sync(F, h1 ? a1 : a4, H1);
  k2 += __shfl_xor_sync(F, h1 ? a2 : a5, H1);
  float m = h2 ? k1 : k0;  // kept: the first or the second of the three
  m += __shfl_xor_sync(F, h2 ? k0 : k1, H2);
  k2 += __shfl_xor_sync(F, k2, H2);
  float r = h3 ? k2 : m;   // kept: that one, or the third
  r += __shfl_xor_sync(F, h3 ? m : k2, H3);
#pragma unroll
  for (int off = H3 / 2; off >= 1; off >>= 1) r += __shfl_xor_sync(F, r, off);
  const int lead = lane & ~(S - 1);
  a0 = __shfl_sync(F, r, lead);
  a1 = __shfl_sync(F, r, lead + H2);
  a2 = __shfl_sync(F, r, lead + H3);
  a3 = __shfl_sync(F, r, lead + H1);
  a4 = __shfl_sync(F, r, lead + H1 + H2);
  a5 = __shfl_sync(F, r, lead + H1 + H3);
}

__device__ __forceinline__ int find_segment(const KParams& p, int tile) {
  int lo = 0, hi = p.n_segs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(p.seg_tile + mid) <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Pair term of one (bead, receptor bead) list entry, branch-free: adds the
// energy to e and returns dE/dx; a pair that is out of range (beyond the
// plateau, bad type) adds 0 energy and returns a zero gradient.
// The bead's ligand type is valid here: phase A gives a bead list entries only
// when its type is inside the pair table.  NE: accumulate the energy too (the
// minimiser's steps before the last need only the gradient).
template <bool NE, bool REF>
__device__ __forceinline__ void pair_term_masked(const KParams& p, const KGrid& G, const BeadPos& bp,
                                                 const float4& r, bool jok, float& e, float& gx, float& gy,
                                                 float& gz) {
  const float dx = bp.x - r.x, dy = bp.y - r.y, dz = bp.z - r.z;
  const float dsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const int rt = __float_as_int(r.w);
  const bool hit = (dsq < G.plateau2) & ((unsigned)rt < (unsigned)G.n_rtypes) & jok;
  const int idx = hit ? bp.lt * G.n_rtypes + rt : 0;
  float4 p0, p1;  // rc, ac, emin, rmin2 / ivor, eplat, gplat, rcap2: one 32-B row
  ldg_f4x2(G.pair + (size_t)(unsigned)idx * 2, p0, p1);
  const float d2 = fmaxf(dsq, p1.w);
  float rr2;  // approximate reciprocal (1 ulp): the pair energy carries ~4 ulp
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rr2) : "f"(d2));
  const float rr6 = rr2 * rr2 * rr2;
  const bool near = d2 < p0.w;
  if (NE) {
    const float vlj = fmaf(p0.x, rr2, -p0.y) * rr6;
    const float en = near ? fmaf(p1.x - 1.f, p0.z, vlj) : p1.x * vlj;
    e += hit ? en - p1.y : 0.f;
  }
  // 2 dnonbon/d(d^2): the factor 2 of d(d^2)/dx folded into the constants
  const float dv2 = rr6 * rr2 * fmaf(-8.f * p0.x, rr2, 6.f * p0.y);
  float gm2 = near ? dv2 : p1.x * dv2;
  gm2 = (dsq < p1.w) ? 0.f : gm2;
  if (REF) {  // the plateau shift's gradient, 1/d with a flush-to-zero approximate rsqrt
    float rd;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rd) : "f"(dsq));
    gm2 = fmaf(-p1.z * G.plateau_x2, rd, gm2);
  }
  const float gf = hit ? gm2 : 0.f;
  gx = gf * dx;
  gy = gf * dy;
  gz = gf * dz;
}

// Blocks of 128 threads per SM: one bead per lane with 32-lane teams runs 6
// (80 registers, one pair in flight per lane), with 8/16-lane teams 5 (their
// minimiser would spill at 80); two beads per lane 4, more 2.  Measured on
// 18-30-bead ligands against a 2500-bead receptor: 6 blocks with one pair in flight beat 5 blocks with
// two by 6 %; with two beads per lane, one pair in flight lost 7-14 %.
template <int S, int K>
__host__ __device__ constexpr int score_blocks_per_sm() { return K == 1 ? (S == 32 ? 6 : 5) : K == 2 ? 4 : 2; }

template <int S, int K, int MODE>
__global__ void __launch_bounds__(128, (score_blocks_per_sm<S, K>())) score_kernel(const __grid_constant__ KParams p) {
  constexpr int P = 32 / S;      // poses per warp
  constexpr int NB = S * K;      // bead slots per pose
  constexpr int U = K == 1 ? 1 : 2;  // pair slots in flight per lane
  constexpr int PB = pairs_per_bead(K) * NB;  // pair-buffer window of one team
  constexpr bool MAT = (MODE == MODE_EVAL_MAT);
  constexpr bool QUAT = (MODE == MODE_QUAT);   // quaternion + adabelief SCHEMA protocol
  constexpr bool ACC9 = MAT || QUAT;           // accumulate dE/dmat (ligand-frame lever arms)
  extern __shared__ __align__(128) unsigned char smem_raw[];

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int slot = lane / S;
  const int tl = lane % S;
  const int lead = slot * S;
  const int RS = rec_stride(p.rec_slot);
  unsigned char* wsm = smem_raw + (size_t)warp * warp_smem_bytes(K, p.rec_slot, ACC9);
  float4* bricks = reinterpret_cast<float4*>(wsm);                          // [32K][8]
  unsigned char* nrec = wsm + 32 * K * 128;                                 // [32K][RS]
  BeadPos* bpos = reinterpret_cast<BeadPos*>(nrec + 32 * K * RS);
  BeadArm* barm = reinterpret_cast<BeadArm*>(nrec + 32 * K * (RS + 16));  // ACC9 modes only
  constexpr int ARM_BYTES = ACC9 ? 16 : 0;
  uint32_t* pbuf = reinterpret_cast<uint32_t*>(nrec + 32 * K * (RS + 16 + ARM_BYTES));
  const int tbase = slot * NB;  // this team's first bead record
  const bool ref_grad = p.grad_mode == ATT_GRAD_REFERENCE;  // the pair loop and phase D compiled per mode
  uint32_t* pb = pbuf + slot * (PB + S);  // this team's pair buffer

  // Grid descriptors: copied from the parameters into shared memory with static
  // parameter offsets only, so that the per-segment grid is picked by a
  // dynamic index into shared memory (never into the parameter space).
  __shared__ KGrid s_grid[ATT_MAX_GRIDS];
#pragma unroll
  for (int g = 0; g < ATT_MAX_GRIDS; ++g)
    if (threadIdx.x == g) s_grid[g] = p.grid[g];
  __syncthreads();


  // statistics (MODE_MIN): bead evaluations with a brick, list lookups, list
  // entries, brick copies, record copies
  // Only the 32-lane kernel with one bead per lane keeps them in registers;
  // the other shapes add warp sums to the counters every step instead (in
  // statistics launches only), which leaves their registers to the step.
  constexpr bool STATS_REGS = (S == 32 && K == 1);
  unsigned c_grid = 0, c_look = 0, c_ent = 0, c_cpb = 0, c_cpr = 0;
  const bool want_stats = p.stats != nullptr;

  int tile;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  if (p.counter != nullptr) {
    int t0 = 0;
    if (lane == 0) t0 = atomicAdd(p.counter, 1);
    tile = __shfl_sync(0xffffffffu, t0, 0);
  } else {
    tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  }

  while (tile < p.n_tiles) {
    const int si = find_segment(p, tile);
    AttSegment sg = p.segs[si];
    // Caller-provided tables are checked before any access they index: the
    // segment's grid, ligand and pose range, the pose's conformer index and
    // the ligand's bead range.  A pose that fails is skipped (no output) and
    // flagged in the device error word.
    const bool seg_ok = ((unsigned)sg.grid < (unsigned)p.n_grids) & ((unsigned)sg.lig < (unsigned)p.n_lig) &
                        (sg.pose0 >= 0) & (sg.n_poses >= 0) &
                        ((long long)sg.pose0 + sg.n_poses <= (long long)p.n_pose_rows);
    const int local = (tile - __ldg(p.seg_tile + si)) * P + slot;
    bool valid = seg_ok & (local >= 0) & (local < sg.n_poses);
    bool bad = !seg_ok;
    if (!seg_ok) sg.grid = sg.lig = sg.pose0 = sg.step0 = 0;
    const int b = sg.pose0 + (valid ? local : 0);
    const KGrid& G = s_grid[sg.grid];
    int lig = sg.lig;
    if (p.pose_lig != nullptr && valid) {
      lig += __ldg(p.pose_lig + b);
      if ((unsigned)lig >= (unsigned)p.n_lig) {
        valid = false;
        bad = true;
        lig = 0;
      }
    }
    const int loff = __ldg(p.lig_off + lig);
    int Ntot = valid ? __ldg(p.lig_off + lig + 1) - loff : 0;
    if (valid && ((loff < 0) | (Ntot < 0) | (Ntot > p.max_beads) | ((long long)loff + Ntot > p.n_lig_beads))) {
      valid = false;
      bad = true;
      Ntot = 0;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&g_kernel_error, ATT_KERR_BAD_SEGMENT);
    // ligands larger than the team's NB bead slots are evaluated in chunks of
    // NB beads; the chunk count is warp-uniform (the chunk loop holds warp
    // barriers and shuffles)
    const int nchunk = __reduce_max_sync(0xffffffffu, (unsigned)((Ntot + NB - 1) / NB));
    const bool multi = nchunk > 1;

    // owned ligand beads (ligand frame), resident for the whole tile
    float lx[K], ly[K], lz[K];
    int ltw[K];
    auto load_beads = [&](int c0) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int i = c0 + tl + k * S;
        if (i < Ntot) {
          const float4 bd = ldg_f4(p.lig_beads + loff + i);
          lx[k] = bd.x; ly[k] = bd.y; lz[k] = bd.z;
          ltw[k] = __float_as_int(bd.w);
        } else {
          lx[k] = ly[k] = lz[k] = 0.f;
          ltw[k] = -1;
        }
      }
    };
    load_beads(0);
    // what this lane's shared-memory slots hold: brick index and record grid
    // point per owned bead (-1: nothing valid).  A bead moves ~0.1 A per ADAM
    // step against 0.9 A cells, so most steps find both still in place.
    int held_b[K], held_v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) held_b[k] = held_v[k] = -1;

    // pose state: team lane k < 6 owns DOF k
    float my_x = 0.f, my_m = 0.f, my_v = 0.f;
    float mat[12];
    if (MAT) {
#pragma unroll
      for (int k = 0; k < 12; ++k)
        mat[k] = valid ? __ldg(p.pose_in + (long long)b * 16 + (k / 3) * 4 + (k % 3)) : 0.f;
    } else if (QUAT) {  // lanes 0..6: qx, qy, qz, qw (scalar last), tx, ty, tz; moments start at 0
      if (valid && tl < 7) my_x = __ldg(p.pose_in + (long long)b * 8 + tl);
    } else if (valid && tl < 6) {
      my_x = __ldg(p.pose_in + (long long)b * 6 + tl);
      if (MODE == MODE_MIN && p.adam != nullptr) {
        my_m = p.adam[(long long)b * 12 + tl];
        my_v = p.adam[(long long)b * 12 + 6 + tl];
      }
    }
    const float dLdE = (MODE == MODE_BWD && valid) ? __ldg(p.dLdE + b) : 0.f;
    int status = 0;
    // a non-finite input pose is flagged (it places no bead on a grid)
    if (MAT) {
#pragma unroll
      for (int k = 0; k < 12; ++k)
        if (!isfinite(mat[k])) status |= ATT_STATUS_NONFINITE_POSE;
    } else {
      const unsigned team = (S == 32) ? 0xffffffffu : (((1u << S) - 1u) << lead);
      if (__ballot_sync(0xffffffffu, valid && tl < (QUAT ? 7 : 6) && !isfinite(my_x)) & team)
        status |= ATT_STATUS_NONFINITE_POSE;
    }
    // quaternion protocol: normalise the input quaternion (Rotation.from_quat),
    // then track the SCHEMA stage, its epoch count and bias-correction powers
    auto normalise_quat = [&]() {
      const float a0 = __shfl_sync(0xffffffffu, my_x, lead + 0), a1 = __shfl_sync(0xffffffffu, my_x, lead + 1);
      const float a2 = __shfl_sync(0xffffffffu, my_x, lead + 2), a3 = __shfl_sync(0xffffffffu, my_x, lead + 3);
      const float n = sqrtf(fmaf(a0, a0, fmaf(a1, a1, fmaf(a2, a2, a3 * a3))));
      if (tl < 4) my_x = my_x / n;
    };
    int stage = 0, k_stage = 0;  // current stage and epochs taken in it
    int st_epochs = 0, st_grav = 0;
    float st_lr = 0.f;
    float last_E = 0.f;          // energy of the latest evaluation (reported, test5.py:465)
    // the values of stage `st` (static parameter indices only: the tables stay
    // in the constant bank, never indexed dynamically in parameter space)
    auto load_stage = [&](int st) {
      st_epochs = 0;
      st_lr = 0.f;
      st_grav = 0;
#pragma unroll
      for (int i = 0; i < ATT_MAX_STAGES; ++i)
        if (i == st) {
          st_epochs = p.qs_epochs[i];
          st_lr = p.qs_lr[i];
          st_grav = p.qs_grav[i];
        }
    };
    if (QUAT) {
      normalise_quat();
      load_stage(stage);
      while (stage < p.qs_n && st_epochs == 0) load_stage(++stage);
    }
    const int nsteps = (MODE == MODE_MIN || QUAT) ? p.steps : 0;  // QUAT: total epochs
    double bp1 = 1.0, bp2 = 1.0;  // beta1^t, beta2^t of the ADAM bias correction
    const int step0 = p.step0 + sg.step0;
    if (MODE == MODE_MIN && step0 > 0) {
      bp1 = pow((double)p.b1, (double)step0);
      bp2 = pow((double)p.b2, (double)step0);
    }

    for (int s = 0; s <= nsteps; ++s) {
      // ---------------- pose -> rotation Q (column form) and translation t
      float q00, q01, q02, q10, q11, q12, q20, q21, q22, tx, ty, tz;
      float sphi = 0.f, cphi = 1.f, spsi = 0.f, cpsi = 1.f;
      float qx = 0.f, qy = 0.f, qz = 0.f, qw = 1.f;  // QUAT: the pose's quaternion
      if (MAT) {
        q00 = mat[0]; q10 = mat[1]; q20 = mat[2];
        q01 = mat[3]; q11 = mat[4]; q21 = mat[5];
        q02 = mat[6]; q12 = mat[7]; q22 = mat[8];
        tx = mat[9]; ty = mat[10]; tz = mat[11];
      } else if (QUAT) {
        // the row-vector matrix of Rotation.as_matrix (homogeneous quaternion
        // form, test5.py:413); column-form Q is its transpose
        qx = __shfl_sync(0xffffffffu, my_x, lead + 0);
        qy = __shfl_sync(0xffffffffu, my_x, lead + 1);
        qz = __shfl_sync(0xffffffffu, my_x, lead + 2);
        qw = __shfl_sync(0xffffffffu, my_x, lead + 3);
        const float x = qx, y = qy, z = qz, w = qw;
        tx = __shfl_sync(0xffffffffu, my_x, lead + 4);
        ty = __shfl_sync(0xffffffffu, my_x, lead + 5);
        tz = __shfl_sync(0xffffffffu, my_x, lead + 6);
        q00 = x * x - y * y - z * z + w * w;  // M00
        q11 = -x * x + y * y - z * z + w * w;  // M11
        q22 = -x * x - y * y + z * z + w * w;  // M22
        q10 = 2.f * (x * y - z * w);           // M01
        q20 = 2.f * (x * z + y * w);           // M02
        q01 = 2.f * (x * y + z * w);           // M10
        q21 = 2.f * (y * z - x * w);           // M12
        q02 = 2.f * (x * z - y * w);           // M20
        q12 = 2.f * (y * z + x * w);           // M21
      } else {
        // team lanes 0..2 hold the three angles: one sincosf per lane, then
        // broadcast (one sincos instruction stream per warp instead of three)
        float my_s, my_c;
        sincosf(my_x, &my_s, &my_c);
        sphi = __shfl_sync(0xffffffffu, my_s, lead + 0);
        cphi = __shfl_sync(0xffffffffu, my_c, lead + 0);
        spsi = __shfl_sync(0xffffffffu, my_s, lead + 1);
        cpsi = __shfl_sync(0xffffffffu, my_c, lead + 1);
        const float sth = __shfl_sync(0xffffffffu, my_s, lead + 2);
        const float cth = __shfl_sync(0xffffffffu, my_c, lead + 2);
        tx = __shfl_sync(0xffffffffu, my_x, lead + 3);
        ty = __shfl_sync(0xffffffffu, my_x, lead + 4);
        tz = __shfl_sync(0xffffffffu, my_x, lead + 5);
        // Q = Rz(phi) Ry(psi) Rz(-theta)
        q00 = cphi * cpsi * cth + sphi * sth;
        q01 = cphi * cpsi * sth - sphi * cth;
        q02 = cphi * spsi;
        q10 = sphi * cpsi * cth - cphi * sth;
        q11 = sphi * cpsi * sth + cphi * cth;
        q12 = sphi * spsi;
        q20 = -spsi * cth;
        q21 = -spsi * sth;
        q22 = cpsi;
      }

      // the energy is needed by every evaluation of the single-evaluation
      // modes, and by the last evaluation of a minimisation (the one reported)
      const bool need_e = (MODE != MODE_MIN && !QUAT) || (MODE == MODE_MIN && s == nsteps) ||
                          (QUAT && s + 1 >= nsteps);
      float acc_e = 0.f, acc_gx = 0.f, acc_gy = 0.f, acc_gz = 0.f;
      float acc_t[ACC9 ? 9 : 3];
#pragma unroll
      for (int k = 0; k < (ACC9 ? 9 : 3); ++k) acc_t[k] = 0.f;

      for (int chunk = 0; chunk < nchunk; ++chunk) {
      const int c0 = chunk * NB;
      const int N = max(0, min(Ntot - c0, NB));  // beads of this chunk
      if (multi) load_beads(c0);
      // ---------------- phase A: move beads, start brick copies, list headers
      float fx[K], fy[K], fz[K], gscale[K];
      int brick_gt[K], bix[K], biy[K], biz[K];  // grid slot, base voxel (for the adjoint scatter)
      bool use[K], outer_k[K];
      int bidx[K];  // brick index (< 2^31: checked on the host)
      int nvox[K];  // nearest list-grid point for the list lookup, -1 = none (< 2^31: checked on the host)
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int i = tl + k * S;
        const bool live = i < N;
        const float rx = fmaf(q00, lx[k], fmaf(q01, ly[k], q02 * lz[k]));
        const float ry = fmaf(q10, lx[k], fmaf(q11, ly[k], q12 * lz[k]));
        const float rz = fmaf(q20, lx[k], fmaf(q21, ly[k], q22 * lz[k]));
        const float X = rx + tx, Y = ry + ty, Z = rz + tz;
        const int gt = ltw[k] & 0xffff, lt = (ltw[k] >> 16) & 0xffff;
        const float vx = (X - G.ox) * G.inv_s;
        const float vy = (Y - G.oy) * G.inv_s;
        const float vz = (Z - G.oz) * G.inv_s;
        const bool inn = live & (vx >= 0.f) & (vx < G.fdx1) & (vy >= 0.f) & (vy < G.fdy1) & (vz >= 0.f) &
                         (vz < G.fdz1);
        bool u = false;
        float ux = vx, uy = vy, uz = vz;
        float sc = G.inv_s;
        int ny = G.dy, nz = G.dz;
        int base = 0;
        outer_k[k] = false;
        if (live && G.bricks != nullptr && gt < G.n_types) {
          u = inn;
          if (!inn && G.has_outer) {
            ux = (vx + G.ext) * 0.5f;
            uy = (vy + G.ext) * 0.5f;
            uz = (vz + G.ext) * 0.5f;
            u = (ux >= 0.f) & (ux < G.fex1) & (uy >= 0.f) & (uy < G.fey1) & (uz >= 0.f) & (uz < G.fez1);
            sc = 0.5f * G.inv_s;
            ny = G.dy2;
            nz = G.dz2;
            base = (int)G.n_inner;
            outer_k[k] = true;
          }
        }
        const float flx = floorf(ux), fly = floorf(uy), flz = floorf(uz);
        fx[k] = ux - flx;
        fy[k] = uy - fly;
        fz[k] = uz - flz;
        gscale[k] = sc;
        // reference floor/ceil weights vanish on an exactly integer coordinate
        if (u && p.quirk && ((fx[k] == 0.f) | (fy[k] == 0.f) | (fz[k] == 0.f))) u = false;
        use[k] = u;
        brick_gt[k] = gt;
        bix[k] = (int)flx;
        biy[k] = (int)fly;
        biz[k] = (int)flz;
        bidx[k] = u ? gt * (int)G.type_stride + base + (bix[k] * (ny - 1) + biy[k]) * (nz - 1) + biz[k] : 0;
        nvox[k] = -1;
        if (inn && G.nb_rec != nullptr && lt < G.n_ltypes && G.n_rec > 0) {
          // nearest list-grid point (the inner grid point itself when nb_scale = 1)
          const int nx = (int)floorf(fmaf(vx, G.nb_scale, 0.5f)), my = (int)floorf(fmaf(vy, G.nb_scale, 0.5f)),
                    mz = (int)floorf(fmaf(vz, G.nb_scale, 0.5f));
          nvox[k] = (nx * G.ndy + my) * G.ndz + mz;
        }
        if (use[k] && !ATT_CHECK(bidx[k] >= 0 && bidx[k] < G.n_bricks, 1, bidx[k], G.n_bricks)) use[k] = false;
        if (nvox[k] >= 0 && !ATT_CHECK(nvox[k] < G.n_vox, 2, nvox[k], G.n_vox)) nvox[k] = -1;
        // records for the team (generic-proxy writes)
        if (live) {
          BeadPos bp;
          bp.x = X; bp.y = Y; bp.z = Z; bp.lt = lt;
          bpos[tbase + i] = bp;
          if (ACC9) {
            BeadArm ba;
            ba.x = lx[k]; ba.y = ly[k]; ba.z = lz[k];
            ba.pad = 0.f;
            barm[tbase + i] = ba;
          }
        }
      }
      // A copy of each brick and neighbour record whose slot does not already
      // hold it (chunked ligands share the slots: always copy); a warp whose
      // slots are all current skips the copy round.
      if (multi) {
#pragma unroll
        for (int k = 0; k < K; ++k) held_b[k] = held_v[k] = -1;
      }
      bool need_b[K], need_v[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        need_b[k] = use[k] && bidx[k] != held_b[k];
        need_v[k] = nvox[k] >= 0 && nvox[k] != held_v[k];
        if (MODE == MODE_MIN && STATS_REGS && want_stats) {
          c_grid += use[k] ? 1u : 0u;
          c_look += nvox[k] >= 0 ? 1u : 0u;
          c_cpb += need_b[k] ? 1u : 0u;
          c_cpr += need_v[k] ? 1u : 0u;
        }
      }
      if (MODE == MODE_MIN && !STATS_REGS && want_stats) {
        unsigned n4[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < K; ++k) {
          n4[0] += use[k] ? 1u : 0u;
          n4[1] += nvox[k] >= 0 ? 1u : 0u;
          n4[2] += need_b[k] ? 1u : 0u;
          n4[3] += need_v[k] ? 1u : 0u;
        }
        const int slot_of[4] = {0, 1, 3, 4};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const unsigned w = __reduce_add_sync(0xffffffffu, n4[i]);
          if (lane == 0 && w) atomicAdd(p.stats + slot_of[i], (unsigned long long)w);
        }
      }
      // The minimisers copy for a few percent of their beads per step: each lane
      // that needs a brick or record copies it (16-byte cp.async through L2,
      // in parallel with the other lanes that copy) and waits for its own
      // copies, and only the owner reads a slot.  Bricks and records are
      // committed as two groups: phase D waits for the first, phase C after it
      // for the second (measured: 3.6 % faster on 18-30-bead ligands against a
      // 2500-bead receptor, 3.8 % on a 40-bead ligand against 5000 beads,
      // and the two phases' values no longer share live registers: the
      // 32-lane minimiser's spills fell from 20 to 4 bytes).  The single-evaluation modes
      // copy for nearly every bead: the warp's copies are listed as (source
      // index, bead slot) in the pair buffer (unused until phase C) and spread
      // over all 32 lanes, consecutive lanes copying consecutive 16-byte chunks
      // of one brick or record, so that a copy instruction fills whole 128-byte
      // lines instead of one chunk of 32 lines; each lane waits for its own
      // copies, and the warp barrier after the wait hands every slot to its
      // owner.  (Listing in the minimisers costs them registers and spills:
      // 14 % slower on 18-30-bead ligands; one chunk of 32 lines per instruction costs
      // the single-evaluation modes a factor 1.9.)  The grid is warp-uniform:
      // a warp's teams share one segment.
      if constexpr (MODE == MODE_MIN || QUAT) {
        unsigned my_bytes = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) my_bytes |= (need_b[k] ? 1u : 0u) | (need_v[k] ? 1u : 0u);
        if (__any_sync(0xffffffffu, my_bytes != 0u)) {
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const unsigned sk = (unsigned)(tbase + tl + k * S);
            if (need_b[k]) {
              const char* src = reinterpret_cast<const char*>(G.bricks + (size_t)bidx[k] * 8);
              const uint32_t dst = smem_u32(bricks) + sk * 128u;
              if constexpr (K == 1) {  // (unrolled, more beads per lane would spill)
#pragma unroll
                for (unsigned c = 0; c < 128u; c += 16u) cp16(dst + c, src + c);
              } else {
#pragma unroll 1
                for (unsigned c = 0; c < 128u; c += 16u) cp16(dst + c, src + c);
              }
              held_b[k] = bidx[k];
            }
          }
          cp_commit();  // group 1: the bricks (phase D waits for it)
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const unsigned sk = (unsigned)(tbase + tl + k * S);
            if (need_v[k]) {
              const unsigned char* src = G.nb_rec + (size_t)nvox[k] * G.nb_rec_bytes;
              const uint32_t dst = smem_u32(nrec) + sk * (unsigned)RS;
              unsigned c0 = 0;
              if constexpr (K == 1) {  // records hold 32, 64 or 128 bytes
                cp16(dst, src);
                cp16(dst + 16u, src + 16);
                c0 = 32u;
              }
#pragma unroll 1
              for (unsigned c = c0; c < (unsigned)G.nb_rec_bytes; c += 16u) cp16(dst + c, src + c);
              held_v[k] = nvox[k];
            }
          }
          cp_commit();  // group 2: the records (phase C waits for it, after phase D)
        }
      } else {
        uint2* list_b = reinterpret_cast<uint2*>(pbuf);  // [32K] bricks
        uint2* list_v = list_b + 32 * K;                 // [32K] records
        unsigned nb_cp = 0, nv_cp = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const unsigned sk = (unsigned)(tbase + tl + k * S);
          const unsigned mb = __ballot_sync(0xffffffffu, need_b[k]);
          const unsigned mv = __ballot_sync(0xffffffffu, need_v[k]);
          if (need_b[k]) {
            list_b[nb_cp + __popc(mb & lanemask_lt())] = make_uint2((unsigned)bidx[k], sk);
            held_b[k] = bidx[k];
          }
          if (need_v[k]) {
            list_v[nv_cp + __popc(mv & lanemask_lt())] = make_uint2((unsigned)nvox[k], sk);
            held_v[k] = nvox[k];
          }
          nb_cp += __popc(mb);
          nv_cp += __popc(mv);
        }
        if (nb_cp + nv_cp != 0u) {
          __syncwarp();
          const char* gb = reinterpret_cast<const char*>(G.bricks);
          for (unsigned i = lane; i < nb_cp * 8u; i += 32u) {
            const uint2 e = list_b[i >> 3];
            const unsigned c = (i & 7u) * 16u;
            cp16(smem_u32(bricks) + e.y * 128u + c, gb + ((size_t)e.x * 128u + c));
          }
          if (nv_cp != 0u) {
            const unsigned RB = (unsigned)G.nb_rec_bytes;  // 32, 64 or 128
            const int rsh = __ffs(RB) - 5;                 // log2 of the 16-byte chunks per record
            for (unsigned i = lane; i < (nv_cp << rsh); i += 32u) {
              const uint2 e = list_v[i >> rsh];
              const unsigned c = (i & ((1u << rsh) - 1u)) * 16u;
              cp16(smem_u32(nrec) + e.y * (unsigned)RS + c, G.nb_rec + ((size_t)e.x * RB + c));
            }
          }
          cp_commit_wait();
          __syncwarp();
        }
      }

      // the minimisers: this lane's bricks have landed (its records may still
      // be in flight while phase D runs)
      if constexpr (MODE == MODE_MIN || QUAT) cp_wait<1>();

      // ---------------- phase D: grid term from the bricks in shared memory
      auto phase_d = [&](auto ne, auto ref) {
      constexpr bool NE = decltype(ne)::value;
      constexpr bool REF = decltype(ref)::value;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (use[k]) {
          const float4* br = bricks + (size_t)(tbase + tl + k * S) * 8;
          float eb = 0.f, gbx = 0.f, gby = 0.f, gbz = 0.f;
          const float sc = gscale[k];
          // Step q reads corner c = q ^ r (r = tl & 7): the 8 lanes of a bank
          // phase read 8 different 16-B bank groups of their 128-B bricks, and
          // the corner's x/y/z offsets are q's static bits flipped by r's, so
          // each weight is a compile-time choice between two per-bead values.
          const int r = tl & 7;
          const int rx = (r >> 2) & 1, ry = (r >> 1) & 1, rz = r & 1;
          const float wx0 = rx ? fx[k] : 1.f - fx[k], wx1 = rx ? 1.f - fx[k] : fx[k];  // q bit 0 / 1
          const float wy0 = ry ? fy[k] : 1.f - fy[k], wy1 = ry ? 1.f - fy[k] : fy[k];
          const float wz0 = rz ? fz[k] : 1.f - fz[k], wz1 = rz ? 1.f - fz[k] : fz[k];
          const float sx0 = rx ? 1.f : -1.f, sy0 = ry ? 1.f : -1.f, sz0 = rz ? 1.f : -1.f;  // d(weight)/d(frac)
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int c = q ^ r;
            const float4 v = br[c];
            const float wx = (q & 4) ? wx1 : wx0, wy = (q & 2) ? wy1 : wy0, wz = (q & 1) ? wz1 : wz0;
            const float w = wx * wy * wz;
            if (NE) eb = fmaf(w, v.x, eb);
            if (REF) {
              gbx = fmaf(-w, v.y, gbx);
              gby = fmaf(-w, v.z, gby);
              gbz = fmaf(-w, v.w, gbz);
            } else {
              const float ce = v.x * sc;
              const float sx = (q & 4) ? -sx0 : sx0, sy = (q & 2) ? -sy0 : sy0, sz = (q & 1) ? -sz0 : sz0;
              gbx = fmaf(ce, sx * wy * wz, gbx);
              gby = fmaf(ce, wx * sy * wz, gby);
              gbz = fmaf(ce, wx * wy * sz, gbz);
            }
            if (MODE == MODE_BWD) {
              const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
              float* dg = outer_k[k] ? p.dgrid_outer : p.dgrid_inner;
              if (dg != nullptr) {
                const int nx = outer_k[k] ? G.dx2 : G.dx;
                const int ny = outer_k[k] ? G.dy2 : G.dy;
                const int nz = outer_k[k] ? G.dz2 : G.dz;
                const long long off =
                    ((((long long)brick_gt[k] * nx + bix[k] + cx) * ny + biy[k] + cy) * (long long)nz + biz[k] + cz) * 4;
                const long long lim = outer_k[k] ? p.n_dgrid_outer : p.n_dgrid_inner;
                if (ATT_CHECK(off >= 0 && off + 4 <= lim, 5, off, lim)) atomicAdd(dg + off, dLdE * w);
              }
            }
          }
          BeadArm ba;  // moment arm: the bead position X, as in the pair term (ACC9: ligand-frame x)
          if (ACC9) {
            ba = barm[tbase + tl + k * S];
          } else {
            const BeadPos bq = bpos[tbase + tl + k * S];
            ba.x = bq.x; ba.y = bq.y; ba.z = bq.z;
          }
          if (NE) acc_e += eb;
          acc_gx += gbx;
          acc_gy += gby;
          acc_gz += gbz;
          if (ACC9) {
            acc_t[0] = fmaf(ba.x, gbx, acc_t[0]); acc_t[1] = fmaf(ba.x, gby, acc_t[1]); acc_t[2] = fmaf(ba.x, gbz, acc_t[2]);
            acc_t[3] = fmaf(ba.y, gbx, acc_t[3]); acc_t[4] = fmaf(ba.y, gby, acc_t[4]); acc_t[5] = fmaf(ba.y, gbz, acc_t[5]);
            acc_t[6] = fmaf(ba.z, gbx, acc_t[6]); acc_t[7] = fmaf(ba.z, gby, acc_t[7]); acc_t[8] = fmaf(ba.z, gbz, acc_t[8]);
          } else {
            acc_t[0] = fmaf(ba.y, gbz, fmaf(-ba.z, gby, acc_t[0]));
            acc_t[1] = fmaf(ba.z, gbx, fmaf(-ba.x, gbz, acc_t[1]));
            acc_t[2] = fmaf(ba.x, gby, fmaf(-ba.y, gbx, acc_t[2]));
          }
        }
      }
      };
      auto run_d = [&]() {
        if (ref_grad) {
          if (need_e) phase_d(std::true_type{}, std::true_type{});
          else phase_d(std::false_type{}, std::true_type{});
        } else {
          if (need_e) phase_d(std::true_type{}, std::false_type{});
          else phase_d(std::false_type{}, std::false_type{});
        }
      };
      // Phase D runs first except in the adjoint, whose grid scatter runs after
      // the pair term (measured on a 65 536-pose backward: 0.454 ms against
      // 0.496 ms with phase D first; the forward modes gain 2 % with it first).
      if constexpr (MODE != MODE_BWD) run_d();
      // the minimisers: this lane's records have landed
      if constexpr (MODE == MODE_MIN || QUAT) cp_wait<0>();
      auto phase_c = [&]() {

      // ---------------- phase C: neighbour pairs, balanced over the team.
      // C1: every owner lane writes its beads' list entries (inline ones from
      // the shared-memory record, the rest from the CSR overflow) as
      // (receptor bead | bead slot << 16) words into the team's pair buffer,
      // runs in lane order.  C2: the team's lanes take the buffered pairs
      // round-robin, U in flight, and add energy, force and torque per pair.
      // Teams with more pairs than the buffer holds take several windows.
      {
        const unsigned ninl = (unsigned)G.nb_inline;
        const int RB = G.nb_rec_bytes;  // record: inline entries, u16 count at RB - 6, u32 overflow at RB - 4
        unsigned ck[K];
        unsigned my_total = 0, my_in = 0;
        bool my_ovf = false;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const unsigned char* rk = nrec + (size_t)(tbase + tl + k * S) * RS;
          ck[k] = (nvox[k] >= 0) ? lds_u16(rk + RB - 6) : 0u;
          my_total += ck[k];
          my_in = max(my_in, min(ck[k], ninl));
          my_ovf |= ck[k] > ninl;
        }
        if (MODE == MODE_MIN && want_stats) {
          if (STATS_REGS) {
            c_ent += my_total;
          } else {
            const unsigned w = __reduce_add_sync(0xffffffffu, my_total);
            if (lane == 0 && w) atomicAdd(p.stats + 2, (unsigned long long)w);
          }
        }
        unsigned incl = my_total;  // inclusive scan over the team's lanes
#pragma unroll
        for (int off = 1; off < S; off <<= 1) {
          const unsigned v = __shfl_up_sync(0xffffffffu, incl, off, S);
          if (tl >= off) incl += v;
        }
        const unsigned team_total = __shfl_sync(0xffffffffu, incl, S - 1, S);
        const unsigned run0 = incl - my_total;  // buffer position of this lane's first entry
        const unsigned warp_max = __reduce_max_sync(0xffffffffu, team_total);
        const unsigned warp_in = __reduce_max_sync(0xffffffffu, my_in);  // longest inline run of the warp
        const bool any_ovf = __any_sync(0xffffffffu, my_ovf);
        for (unsigned q0 = 0; q0 < warp_max; q0 += PB) {
          // inline entries, eight per 16-byte shared load (at the 48-byte
          // stride of 32-byte records each quarter-warp phase is free of bank
          // conflicts); a team whose pairs fit one window (the common case)
          // needs no window test per entry
          const bool one_window = warp_max <= (unsigned)PB;
          for (unsigned c = 0; c < warp_in; c += 8) {
            unsigned r = run0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
              const unsigned nin = min(ck[k], ninl);
              if (c < nin) {
                const unsigned char* rk = nrec + (size_t)(tbase + tl + k * S) * RS;
                const uint4 q = lds_u128(rk + 2 * c);
                const unsigned w[4] = {q.x, q.y, q.z, q.w};
                const unsigned tag = (unsigned)(tl + k * S) << 16;
                // (receptor bead | bead slot << 16): one byte permute per entry
                unsigned v[8];
#pragma unroll
                for (unsigned i = 0; i < 4; ++i) {
                  v[2 * i] = __byte_perm(w[i], tag, 0x7610);
                  v[2 * i + 1] = __byte_perm(w[i], tag, 0x7632);
                }
                if (one_window) {
                  uint32_t* dst = pb + (r + c);
#pragma unroll
                  for (unsigned i = 0; i < 8; ++i)
                    if (c + i < nin) dst[i] = v[i];
                } else {
#pragma unroll
                  for (unsigned i = 0; i < 8; ++i) {
                    const unsigned pos = r + c + i - q0;
                    if ((c + i < nin) & (pos < (unsigned)PB)) pb[pos] = v[i];
                  }
                }
              }
              r += ck[k];
            }
          }
          if (any_ovf) {  // entries beyond the inline ones, from the CSR list
            unsigned r = run0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
              if (ck[k] > ninl) {
                const unsigned char* rk = nrec + (size_t)(tbase + tl + k * S) * RS;
                const unsigned ovf = lds_u32(rk + RB - 4);
                const unsigned tag = (unsigned)(tl + k * S) << 16;
                const unsigned lo = max(q0, r + ninl), hi = min(r + ck[k], q0 + PB);
#ifdef ATT_BOUNDS_CHECK
                if (!ATT_CHECK((long long)ovf - ninl + ck[k] <= G.n_list, 6, ovf, ck[k])) {
                  for (unsigned s = lo; s < hi; ++s) pb[s - q0] = ATT_NB_EMPTY | tag;
                  r += ck[k];
                  continue;
                }
#endif
                for (unsigned s = lo; s < hi; ++s) pb[s - q0] = ldg_nc_u16(G.nb_list + (ovf + (s - r - ninl))) | tag;
              }
              r += ck[k];
            }
          }
          __syncwarp();
          const unsigned n = min(team_total - min(team_total, q0), (unsigned)PB);
          auto pair_window = [&](auto ne, auto ref) {
          constexpr bool NE = decltype(ne)::value;
          constexpr bool REF = decltype(ref)::value;
          for (unsigned s0 = tl; s0 < n; s0 += U * S) {
            unsigned ww[U];
#pragma unroll
            for (int m = 0; m < U; ++m) {
              const unsigned s = s0 + m * S;
              ww[m] = (s < n) ? pb[s] : (unsigned)ATT_NB_EMPTY;
            }
            float4 rr[U];
            bool jok[U];
#pragma unroll
            for (int m = 0; m < U; ++m) {
              const unsigned j = ww[m] & 0xffffu;
#ifdef ATT_BOUNDS_CHECK
              if (j != ATT_NB_EMPTY) (void)ATT_CHECK(j < (unsigned)G.n_rec, 4, j, G.n_rec);
#endif
              // an entry outside the receptor (the empty-slot sentinel) reads the last
              // bead and is masked in the pair term (phase A gives beads list entries
              // only when the receptor has beads)
              jok[m] = j < (unsigned)G.n_rec;
              rr[m] = ldg_f4(G.rec + min(j, (unsigned)G.n_rec - 1u));
            }
#pragma unroll
            for (int m = 0; m < U; ++m) {
              const unsigned bi = tbase + (ww[m] >> 16);
              const BeadPos bp = bpos[bi];
              float px, py, pz;
              pair_term_masked<NE, REF>(p, G, bp, rr[m], jok[m], acc_e, px, py, pz);
              // moment arm: the bead position X (the torque about t, sum (X - t) x g,
              // is sum X x g - t x sum g, formed after the team sum); the
              // 4x4 form accumulates with the ligand-frame x
              BeadArm ba;
              if (ACC9) ba = barm[bi];
              else { ba.x = bp.x; ba.y = bp.y; ba.z = bp.z; }
              acc_gx += px;
              acc_gy += py;
              acc_gz += pz;
              if (ACC9) {
                acc_t[0] = fmaf(ba.x, px, acc_t[0]); acc_t[1] = fmaf(ba.x, py, acc_t[1]); acc_t[2] = fmaf(ba.x, pz, acc_t[2]);
                acc_t[3] = fmaf(ba.y, px, acc_t[3]); acc_t[4] = fmaf(ba.y, py, acc_t[4]); acc_t[5] = fmaf(ba.y, pz, acc_t[5]);
                acc_t[6] = fmaf(ba.z, px, acc_t[6]); acc_t[7] = fmaf(ba.z, py, acc_t[7]); acc_t[8] = fmaf(ba.z, pz, acc_t[8]);
              } else {
                acc_t[0] = fmaf(ba.y, pz, fmaf(-ba.z, py, acc_t[0]));
                acc_t[1] = fmaf(ba.z, px, fmaf(-ba.x, pz, acc_t[1]));
                acc_t[2] = fmaf(ba.x, py, fmaf(-ba.y, px, acc_t[2]));
              }
            }
          }
          };
          if (ref_grad) {
            if (need_e) pair_window(std::true_type{}, std::true_type{});
            else pair_window(std::false_type{}, std::true_type{});
          } else {
            if (need_e) pair_window(std::true_type{}, std::false_type{});
            else pair_window(std::false_type{}, std::false_type{});
          }
          __syncwarp();  // the next window overwrites the buffer
        }
      }
      };
      phase_c();
      if constexpr (MODE == MODE_BWD) run_d();

      // the next chunk's / evaluation's copies (by any lane of the warp)
      // overwrite the slots read above
      __syncwarp();
      }  // chunks

      // ---------------- team reduction and output / ADAM
      if (need_e) acc_e = team_sum<S>(acc_e);
      if constexpr (!ACC9 && (K == 1 || S == 32)) {
        team_sum6<S>(acc_gx, acc_gy, acc_gz, acc_t[0], acc_t[1], acc_t[2], lane);
      } else {
        acc_gx = team_sum<S>(acc_gx);
        acc_gy = team_sum<S>(acc_gy);
        acc_gz = team_sum<S>(acc_gz);
#pragma unroll
        for (int k = 0; k < (ACC9 ? 9 : 3); ++k) acc_t[k] = team_sum<S>(acc_t[k]);
      }
      if (!ACC9) {  // torque about the pose's translation: sum X x g - t x sum g
        acc_t[0] -= fmaf(ty, acc_gz, -tz * acc_gy);
        acc_t[1] -= fmaf(tz, acc_gx, -tx * acc_gz);
        acc_t[2] -= fmaf(tx, acc_gy, -ty * acc_gx);
      }

      if constexpr (QUAT) {
        // ---- SCHEMA protocol step (test5.py:450-458): energy and gradient
        // with this stage's gravity, dE/dq from dE/dM through the quaternion
        // form, optax.adabelief update on lanes 0..6, renormalised quaternion
        const float grav = st_grav ? p.gravity : 0.f;
        last_E = acc_e + grav * (tx * tx + ty * ty + tz * tz);
        const float G00 = acc_t[0], G01 = acc_t[1], G02 = acc_t[2];
        const float G10 = acc_t[3], G11 = acc_t[4], G12 = acc_t[5];
        const float G20 = acc_t[6], G21 = acc_t[7], G22 = acc_t[8];
        const float x = qx, y = qy, z = qz, w = qw;
        const float gqx = 2.f * (G00 * x + G01 * y + G02 * z + G10 * y - G11 * x - G12 * w + G20 * z + G21 * w - G22 * x);
        const float gqy = 2.f * (-G00 * y + G01 * x + G02 * w + G10 * x + G11 * y + G12 * z - G20 * w + G21 * z - G22 * y);
        const float gqz = 2.f * (-G00 * z - G01 * w + G02 * x + G10 * w - G11 * z + G12 * y + G20 * x + G21 * y + G22 * z);
        const float gqw = 2.f * (G00 * w - G01 * z + G02 * y + G10 * z + G11 * w - G12 * x - G20 * y + G21 * x + G22 * w);
        const float gtx = acc_gx + 2.f * grav * tx, gty = acc_gy + 2.f * grav * ty, gtz = acc_gz + 2.f * grav * tz;
        float gk = gqx;
        gk = (tl == 1) ? gqy : gk;
        gk = (tl == 2) ? gqz : gk;
        gk = (tl == 3) ? gqw : gk;
        gk = (tl == 4) ? gtx : gk;
        gk = (tl == 5) ? gty : gk;
        gk = (tl == 6) ? gtz : gk;
        const bool ok = isfinite(gqx) & isfinite(gqy) & isfinite(gqz) & isfinite(gqw) & isfinite(gtx) &
                        isfinite(gty) & isfinite(gtz);
        ++k_stage;
        bp1 *= (double)p.b1;
        bp2 *= (double)p.b2;
        if (!ok) {
          status |= ATT_STATUS_NONFINITE_GRAD;
        } else if (tl < 7) {
          const float err = gk - my_m;  // against the previous first moment (optax scale_by_belief)
          my_m = fmaf(p.b1, my_m, (1.f - p.b1) * gk);
          my_v = fmaf(p.b2, my_v, (1.f - p.b2) * err * err) + p.eps_root;
          // bias-corrected moments; approximate divisions (2 ulp) keep the
          // update off the IEEE division's slow path
          const float mh = __fdividef(my_m, (float)(1.0 - bp1));
          const float vh = __fdividef(my_v, (float)(1.0 - bp2));
          my_x -= __fdividef(st_lr * mh, sqrtf(vh) + p.eps);
        }
        normalise_quat();  // Rotation.from_quat(rotations.as_quat())
        if (k_stage >= st_epochs) {  // next stage: a fresh optimiser state
          load_stage(++stage);
          while (stage < p.qs_n && st_epochs == 0) load_stage(++stage);
          k_stage = 0;
          my_m = my_v = 0.f;
          bp1 = bp2 = 1.0;
        }
        if (s + 1 >= nsteps) break;
        continue;
      }

      const float etot = acc_e + p.gravity * (tx * tx + ty * ty + tz * tz);
      if (MAT) {
        if (valid) {
          if (tl == 0) p.energy[b] = etot;
          if (p.grad != nullptr) {
            for (int k = tl; k < 16; k += S) {
              const int r = k >> 2, c = k & 3;
              float v = 0.f;
              if (c < 3) {
                if (r < 3) v = acc_t[r * 3 + c];
                else v = (c == 0) ? acc_gx + 2.f * p.gravity * tx
                                  : (c == 1 ? acc_gy + 2.f * p.gravity * ty : acc_gz + 2.f * p.gravity * tz);
              }
              p.grad[(long long)b * 16 + k] = v;
            }
          }
          if (tl == 0 && p.status != nullptr) p.status[b] = status | (isfinite(etot) ? 0 : ATT_STATUS_NONFINITE_ENERGY);
        }
        break;
      }
      // pose gradient: dE/dt and dE/d(angle_k) = w_k . torque
      const float gtx = acc_gx + 2.f * p.gravity * tx;
      const float gty = acc_gy + 2.f * p.gravity * ty;
      const float gtz = acc_gz + 2.f * p.gravity * tz;
      const float gphi = acc_t[2];
      const float gpsi = -sphi * acc_t[0] + cphi * acc_t[1];
      const float gth = -(cphi * spsi * acc_t[0] + sphi * spsi * acc_t[1] + cpsi * acc_t[2]);
      float gk = gphi;
      gk = (tl == 1) ? gpsi : gk;
      gk = (tl == 2) ? gth : gk;
      gk = (tl == 3) ? gtx : gk;
      gk = (tl == 4) ? gty : gk;
      gk = (tl == 5) ? gtz : gk;

      if (MODE == MODE_EVAL || MODE == MODE_BWD || s == nsteps) {
        if (!isfinite(etot)) status |= ATT_STATUS_NONFINITE_ENERGY;
        if (valid) {
          if (MODE == MODE_BWD) {
            if (tl < 6 && p.dLdpose != nullptr) p.dLdpose[(long long)b * 6 + tl] = dLdE * gk;
          } else {
            if (tl == 0) p.energy[b] = etot;
            if (MODE == MODE_EVAL && tl < 6 && p.grad != nullptr) p.grad[(long long)b * 6 + tl] = gk;
          }
        }
        break;
      }
      // ---- fused ADAM step on lanes 0..5 (optax.adam form)
      const bool ok = isfinite(gtx) & isfinite(gty) & isfinite(gtz) & isfinite(gphi) & isfinite(gpsi) &
                      isfinite(gth);
      // beta^t as running double products (t counts skipped steps too)
      bp1 *= (double)p.b1;
      bp2 *= (double)p.b2;
      if (!ok) {
        status |= ATT_STATUS_NONFINITE_GRAD;
      } else if (tl < 6) {
        my_m = fmaf(p.b1, my_m, (1.f - p.b1) * gk);
        my_v = fmaf(p.b2, my_v, (1.f - p.b2) * gk * gk);
        // bias-corrected moments; approximate divisions (2 ulp) keep the
        // update off the IEEE division's slow path
        const float mh = __fdividef(my_m, (float)(1.0 - bp1));
        const float vh = __fdividef(my_v, (float)(1.0 - bp2));
        const float lr = (tl < 3) ? p.lr_rot : p.lr_trans;
        float sv;  // approximate square root (the update's divisions are approximate too)
        asm("sqrt.approx.f32 %0, %1;" : "=f"(sv) : "f"(vh));
        my_x -= __fdividef(lr * mh, sv + p.eps);
      }
    }

    if (QUAT && valid) {
      if (tl < 7) p.pose_out[(long long)b * 8 + tl] = my_x;
      if (tl == 0) p.energy[b] = last_E;
      if (!isfinite(last_E)) status |= ATT_STATUS_NONFINITE_ENERGY;
    }
    if (MODE == MODE_MIN && valid && tl < 6) {
      p.pose_out[(long long)b * 6 + tl] = my_x;
      if (p.adam != nullptr) {
        p.adam[(long long)b * 12 + tl] = my_m;
        p.adam[(long long)b * 12 + 6 + tl] = my_v;
      }
    }
    if ((MODE == MODE_MIN || MODE == MODE_EVAL || QUAT) && valid && tl == 0 && p.status != nullptr)
      p.status[b] = status;

    if (p.counter != nullptr) {
      int t0 = 0;
      if (lane == 0) t0 = atomicAdd(p.counter, 1);
      tile = __shfl_sync(0xffffffffu, t0, 0);
    } else {
      tile += nwarps;
    }
  }

  if (MODE == MODE_MIN && STATS_REGS && p.stats != nullptr) {
    unsigned long long v[5] = {c_grid, c_look, c_ent, c_cpb, c_cpr};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
      if (lane == 0 && v[k]) atomicAdd(p.stats + k, v[k]);
    }
  }
}

// ---------------------------------------------------------------------------
// launch plumbing: (S, K) instantiations and their shared-memory needs
// ---------------------------------------------------------------------------
template <int MODE>
struct KernelTable {
  static const void* get(int S, int K) {
#define ATT_CASE(s_, k_) \
  if (S == s_ && K == k_) return (const void*)score_kernel<s_, k_, MODE>;
    ATT_CASE(32, 1) ATT_CASE(32, 2) ATT_CASE(32, 4) ATT_CASE(32, 8)
    ATT_CASE(16, 1) ATT_CASE(16, 2) ATT_CASE(16, 4) ATT_CASE(16, 8)
    ATT_CASE(8, 1) ATT_CASE(8, 2) ATT_CASE(8, 4) ATT_CASE(8, 8)
#undef ATT_CASE
    return nullptr;
  }
};

static const void* kernel_of(int mode, int S, int K) {
  switch (mode) {
    case MODE_EVAL: return KernelTable<MODE_EVAL>::get(S, K);
    case MODE_EVAL_MAT: return KernelTable<MODE_EVAL_MAT>::get(S, K);
    case MODE_MIN: return KernelTable<MODE_MIN>::get(S, K);
    case MODE_BWD: return KernelTable<MODE_BWD>::get(S, K);
    case MODE_QUAT: return KernelTable<MODE_QUAT>::get(S, K);
  }
  return nullptr;
}

int beads_per_lane(int S, int max_beads) {
  const int need = (max_beads + S - 1) / S;
  int K = 1;
  while (K < need) K <<= 1;
  return K <= ATT_MAX_BEADS_PER_LANE ? K : ATT_MAX_BEADS_PER_LANE;  // larger ligands run in chunks
}

size_t score_smem_bytes(int K, int threads, int rec_slot) {
  return warp_smem_bytes(K, rec_slot) * (size_t)(threads / 32);
}

// the shared memory of one block of `mode` (without bead arms unless the mode
// accumulates dE/dmat)
static size_t mode_smem_bytes(int mode, int K, int threads, int rec_slot) {
  const bool arms = mode == MODE_EVAL_MAT || mode == MODE_QUAT;
  return warp_smem_bytes(K, rec_slot, arms) * (size_t)(threads / 32);
}

cudaError_t launch_score(const KParams& p, int mode, int S, int K, int blocks, int threads, cudaStream_t st) {
  const void* k = kernel_of(mode, S, K);
  if (k == nullptr) return cudaErrorInvalidValue;
  const size_t smem = mode_smem_bytes(mode, K, threads, p.rec_slot);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  void* args[] = {const_cast<KParams*>(&p)};
  return cudaLaunchKernel(k, dim3(blocks), dim3(threads), args, smem, st);
}

cudaError_t kernel_status(int* out, int clear, cudaStream_t st) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(out, g_kernel_error, sizeof(int), 0, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && clear && *out) {
    const int zero = 0;
    e = cudaMemcpyToSymbolAsync(g_kernel_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e;
}

cudaError_t kernel_debug_info(unsigned long long* out3, int clear, cudaStream_t st) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(out3, g_kernel_debug, 3 * sizeof(unsigned long long), 0,
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && clear) {
    const unsigned long long zero[3] = {0ull, 0ull, 0ull};
    e = cudaMemcpyToSymbolAsync(g_kernel_debug, zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e;
}

cudaError_t occupancy_blocks(int mode, int S, int K, int threads, int rec_slot, int* blocks_per_sm) {
  const void* k = kernel_of(mode, S, K);
  if (k == nullptr) return cudaErrorInvalidValue;
  const size_t smem = mode_smem_bytes(mode, K, threads, rec_slot);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, smem);
}

}  // namespace att
