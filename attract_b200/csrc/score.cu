// Scoring and fused minimisation kernels (K1 energrad / minimise, K2 adjoint).
//
// One pose is served by a team of S lanes (S = 8, 16 or 32; 32/S poses per
// warp).  A team is split into 8-lane subteams; a subteam takes one ligand bead
// at a time and its 8 lanes cooperate on it:
//   * lane c reads trilinear corner c of the bead's 128-byte grid brick (the 8
//     corners are contiguous, so the subteam issues one coalesced 128-B load),
//   * the lanes stride over the bead's neighbour list (entry c, c+8, ...).
// Energy, dE/dx and the torque are linear in the per-corner / per-pair
// contributions, so every lane accumulates its own share and the team sums its
// 7 accumulators with xor-shuffles once per step.  The rigid-body ADAM update
// of the 6 pose DOFs runs on team lanes 0..5 between steps, the pose never
// leaves registers, and a persistent launch pulls tiles of poses from a work
// counter until all segments are done.
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

#include "common.cuh"

namespace att {

struct BeadAcc {
  float e, gx, gy, gz;   // energy and dE/dx of this lane's share
};

template <int MODE>
struct PoseAcc {
  // energy, dE/dt, then torque (3) or dE/dmat rows (9)
  static constexpr int NT = (MODE == MODE_EVAL_MAT) ? 9 : 3;
  float e, gx, gy, gz;
  float t[NT];
};

// Per-bead work of one subteam lane: grid corner `corner` and list entries
// corner, corner+8, ...  X is the moved bead, (bx,by,bz) its ligand-frame
// coordinates.  `dscale` scales scatter-added grid gradients (MODE_BWD).
template <int MODE>
__device__ __forceinline__ void bead_work(const KParams& p, const KGrid& G, int corner, float X, float Y,
                                          float Z, int gt, int lt, BeadAcc& a, float dscale,
                                          unsigned& c_grid, unsigned& c_look, unsigned& c_ent) {
  const float vx = (X - G.ox) * G.inv_s;
  const float vy = (Y - G.oy) * G.inv_s;
  const float vz = (Z - G.oz) * G.inv_s;
  const bool inn = (vx >= 0.f) & (vx < G.fdx1) & (vy >= 0.f) & (vy < G.fdy1) & (vz >= 0.f) & (vz < G.fdz1);
  if (G.bricks != nullptr && gt < G.n_types) {
    float ux = vx, uy = vy, uz = vz, scale = G.inv_s;
    bool use = inn;
    int ny = G.dy, nz = G.dz;
    long long base = 0;
    if (!inn && G.has_outer) {
      ux = (vx + G.ext) * 0.5f;
      uy = (vy + G.ext) * 0.5f;
      uz = (vz + G.ext) * 0.5f;
      use = (ux >= 0.f) & (ux < G.fex1) & (uy >= 0.f) & (uy < G.fey1) & (uz >= 0.f) & (uz < G.fez1);
      scale = 0.5f * G.inv_s;
      ny = G.dy2;
      nz = G.dz2;
      base = G.n_inner;
    }
    if (use) {
      const float flx = floorf(ux), fly = floorf(uy), flz = floorf(uz);
      const float fx = ux - flx, fy = uy - fly, fz = uz - flz;
      // reference floor/ceil weights vanish on an exactly integer coordinate
      if (p.quirk && ((fx == 0.f) | (fy == 0.f) | (fz == 0.f))) use = false;
      if (use) {
        const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
        const long long brick = (long long)gt * G.type_stride + base +
                                ((long long)ix * (ny - 1) + iy) * (nz - 1) + iz;
        const float4 c = ldg_stream_f4(G.bricks + brick * 8 + corner);
        const int cx = (corner >> 2) & 1, cy = (corner >> 1) & 1, cz = corner & 1;
        const float wx = cx ? fx : 1.f - fx;
        const float wy = cy ? fy : 1.f - fy;
        const float wz = cz ? fz : 1.f - fz;
        const float w = wx * wy * wz;
        a.e = fmaf(w, c.x, a.e);
        if (p.grad_mode == ATT_GRAD_REFERENCE) {
          a.gx = fmaf(-w, c.y, a.gx);
          a.gy = fmaf(-w, c.z, a.gy);
          a.gz = fmaf(-w, c.w, a.gz);
        } else {
          const float ce = c.x * scale;
          a.gx = fmaf(ce, (cx ? 1.f : -1.f) * wy * wz, a.gx);
          a.gy = fmaf(ce, wx * (cy ? 1.f : -1.f) * wz, a.gy);
          a.gz = fmaf(ce, wx * wy * (cz ? 1.f : -1.f), a.gz);
        }
        if (MODE == MODE_BWD) {
          float* dg = base ? p.dgrid_outer : p.dgrid_inner;
          if (dg != nullptr) {
            const int gx = ix + cx, gy = iy + cy, gz = iz + cz;
            const int nx = base ? G.dx2 : G.dx;
            const long long off = ((((long long)gt * nx + gx) * ny + gy) * (long long)nz + gz) * 4;
            atomicAdd(dg + off, dscale * w);
          }
        }
        if (MODE == MODE_MIN && corner == 0) c_grid += 1;
      }
    }
  }
  if (G.nb_hdr != nullptr && inn && lt < G.n_ltypes) {
    const int nx = (int)floorf(vx + 0.5f), ny = (int)floorf(vy + 0.5f), nz = (int)floorf(vz + 0.5f);
    const uint2 h = ldg_u2(G.nb_hdr + (((long long)nx * G.dy + ny) * G.dz + nz));
    if (MODE == MODE_MIN && corner == 0) c_look += 1;
    const float4* prow = G.pair + (long long)lt * G.n_rtypes * 2;
    for (unsigned e = corner; e < h.y; e += 8) {
      const unsigned j = ldg_u16(G.nb_list + h.x + e);
      if (MODE == MODE_MIN) c_ent += 1;
      if (j >= (unsigned)G.n_rec) continue;  // ATT_NB_EMPTY and corrupt entries
      const float4 r = ldg_f4(G.rec + j);
      const float dx = X - r.x, dy = Y - r.y, dz = Z - r.z;
      const float dsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (!(dsq < G.plateau2)) continue;
      const int rt = __float_as_int(r.w);
      if ((unsigned)rt >= (unsigned)G.n_rtypes) continue;
      const float4 p0 = ldg_f4(prow + rt * 2);      // rc, ac, emin, rmin2
      const float4 p1 = ldg_f4(prow + rt * 2 + 1);  // ivor, eplat, gplat, rcap2
      const float d2 = fmaxf(dsq, p1.w);
      const float rr2 = __frcp_rn(d2);
      const float rr6 = rr2 * rr2 * rr2;
      const float vlj = fmaf(p0.x, rr2, -p0.y) * rr6;
      const bool near = d2 < p0.w;
      const float en = near ? fmaf(p1.x - 1.f, p0.z, vlj) : p1.x * vlj;
      const float dv = rr6 * rr2 * fmaf(-4.f * p0.x, rr2, 3.f * p0.y);
      float gm = near ? dv : p1.x * dv;
      if (dsq < p1.w) gm = 0.f;
      a.e += en - p1.y;
      if (p.grad_mode == ATT_GRAD_REFERENCE) gm = fmaf(-p1.z * G.plateau, rsqrtf(dsq), gm);
      const float gf = 2.f * gm;
      a.gx = fmaf(gf, dx, a.gx);
      a.gy = fmaf(gf, dy, a.gy);
      a.gz = fmaf(gf, dz, a.gz);
    }
  }
}

template <int S>
__device__ __forceinline__ float team_sum(float v) {
#pragma unroll
  for (int off = S / 2; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__device__ __forceinline__ int find_segment(const KParams& p, int tile) {
  int lo = 0, hi = p.n_segs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(p.seg_tile + mid) <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int S, int MODE>
__global__ void __launch_bounds__(256) score_kernel(const __grid_constant__ KParams p) {
  constexpr int P = 32 / S;
  constexpr int NSUB = S / 8;
  const int lane = threadIdx.x & 31;
  const int slot = lane / S;
  const int tl = lane % S;
  const int sub = tl >> 3;
  const int corner = lane & 7;
  const int lead = slot * S;  // team lane 0

  unsigned c_grid = 0, c_look = 0, c_ent = 0;  // statistics (MODE_MIN)

  int tile;
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  if (p.counter != nullptr) {
    int t0 = 0;
    if (lane == 0) t0 = atomicAdd(p.counter, 1);
    tile = __shfl_sync(0xffffffffu, t0, 0);
  } else {
    tile = warp_global;
  }

  while (tile < p.n_tiles) {
    const int si = find_segment(p, tile);
    const AttSegment sg = p.segs[si];
    const int local = (tile - __ldg(p.seg_tile + si)) * P + slot;
    const bool valid = local < sg.n_poses;
    const int b = sg.pose0 + (valid ? local : 0);
    const KGrid& G = p.grid[sg.grid];
    int lig = sg.lig;
    if (p.pose_lig != nullptr && valid) lig += __ldg(p.pose_lig + b);
    const int loff = __ldg(p.lig_off + lig);
    const int N = valid ? __ldg(p.lig_off + lig + 1) - loff : 0;

    // ---- pose state: team lane k < 6 owns DOF k ----
    float my_x = 0.f, my_m = 0.f, my_v = 0.f;
    float mat[12];
    if (MODE == MODE_EVAL_MAT) {
#pragma unroll
      for (int k = 0; k < 12; ++k) mat[k] = valid ? __ldg(p.pose_in + (long long)b * 16 + (k / 3) * 4 + (k % 3)) : 0.f;
    } else {
      if (valid && tl < 6) {
        my_x = __ldg(p.pose_in + (long long)b * 6 + tl);
        if (MODE == MODE_MIN && p.adam != nullptr) {
          my_m = p.adam[(long long)b * 12 + tl];
          my_v = p.adam[(long long)b * 12 + 6 + tl];
        }
      }
    }
    const float dLdE = (MODE == MODE_BWD && valid) ? __ldg(p.dLdE + b) : 0.f;
    int status = 0;
    const int nsteps = (MODE == MODE_MIN) ? p.steps : 0;

    for (int s = 0; s <= nsteps; ++s) {
      float q00, q01, q02, q10, q11, q12, q20, q21, q22, tx, ty, tz;
      float sphi = 0.f, cphi = 1.f, spsi = 0.f, cpsi = 1.f;
      if (MODE == MODE_EVAL_MAT) {
        // x'_j = sum_i x_i mat[i][j] + mat[3][j]  ->  Q[j][i] = mat[i][j]
        q00 = mat[0]; q10 = mat[1]; q20 = mat[2];
        q01 = mat[3]; q11 = mat[4]; q21 = mat[5];
        q02 = mat[6]; q12 = mat[7]; q22 = mat[8];
        tx = mat[9]; ty = mat[10]; tz = mat[11];
      } else {
        const float phi = __shfl_sync(0xffffffffu, my_x, lead + 0);
        const float psi = __shfl_sync(0xffffffffu, my_x, lead + 1);
        const float th = __shfl_sync(0xffffffffu, my_x, lead + 2);
        tx = __shfl_sync(0xffffffffu, my_x, lead + 3);
        ty = __shfl_sync(0xffffffffu, my_x, lead + 4);
        tz = __shfl_sync(0xffffffffu, my_x, lead + 5);
        float sth, cth;
        sincosf(phi, &sphi, &cphi);
        sincosf(psi, &spsi, &cpsi);
        sincosf(th, &sth, &cth);
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

      PoseAcc<MODE> acc;
      acc.e = acc.gx = acc.gy = acc.gz = 0.f;
#pragma unroll
      for (int k = 0; k < PoseAcc<MODE>::NT; ++k) acc.t[k] = 0.f;

      for (int i = sub; i < N; i += NSUB) {
        const float4 bd = ldg_f4(p.lig_beads + loff + i);
        const int tw = __float_as_int(bd.w);
        const int gt = tw & 0xffff, lt = (tw >> 16) & 0xffff;
        const float rx = fmaf(q00, bd.x, fmaf(q01, bd.y, q02 * bd.z));
        const float ry = fmaf(q10, bd.x, fmaf(q11, bd.y, q12 * bd.z));
        const float rz = fmaf(q20, bd.x, fmaf(q21, bd.y, q22 * bd.z));
        BeadAcc a = {0.f, 0.f, 0.f, 0.f};
        bead_work<MODE>(p, G, corner, rx + tx, ry + ty, rz + tz, gt, lt, a, dLdE, c_grid, c_look, c_ent);
        acc.e += a.e;
        acc.gx += a.gx;
        acc.gy += a.gy;
        acc.gz += a.gz;
        if (MODE == MODE_EVAL_MAT) {
          // dE/dmat[i][j] = sum_b x_b,i g_b,j
          acc.t[0] = fmaf(bd.x, a.gx, acc.t[0]);
          acc.t[1] = fmaf(bd.x, a.gy, acc.t[1]);
          acc.t[2] = fmaf(bd.x, a.gz, acc.t[2]);
          acc.t[3] = fmaf(bd.y, a.gx, acc.t[3]);
          acc.t[4] = fmaf(bd.y, a.gy, acc.t[4]);
          acc.t[5] = fmaf(bd.y, a.gz, acc.t[5]);
          acc.t[6] = fmaf(bd.z, a.gx, acc.t[6]);
          acc.t[7] = fmaf(bd.z, a.gy, acc.t[7]);
          acc.t[8] = fmaf(bd.z, a.gz, acc.t[8]);
        } else {
          // torque r x g with r = Q x
          acc.t[0] = fmaf(ry, a.gz, fmaf(-rz, a.gy, acc.t[0]));
          acc.t[1] = fmaf(rz, a.gx, fmaf(-rx, a.gz, acc.t[1]));
          acc.t[2] = fmaf(rx, a.gy, fmaf(-ry, a.gx, acc.t[2]));
        }
      }

      acc.e = team_sum<S>(acc.e);
      acc.gx = team_sum<S>(acc.gx);
      acc.gy = team_sum<S>(acc.gy);
      acc.gz = team_sum<S>(acc.gz);
#pragma unroll
      for (int k = 0; k < PoseAcc<MODE>::NT; ++k) acc.t[k] = team_sum<S>(acc.t[k]);

      const float etot = acc.e + p.gravity * (tx * tx + ty * ty + tz * tz);
      if (MODE == MODE_EVAL_MAT) {
        if (valid) {
          if (tl == 0) p.energy[b] = etot;
          if (p.grad != nullptr) {
            for (int k = tl; k < 16; k += S) {
              const int r = k >> 2, c = k & 3;
              float v = 0.f;
              if (c < 3) {
                if (r < 3) v = acc.t[r * 3 + c];
                else v = (c == 0) ? acc.gx : (c == 1 ? acc.gy : acc.gz);
              }
              p.grad[(long long)b * 16 + k] = v;
            }
          }
        }
        break;
      }
      // pose gradient: dE/dt and dE/d(angle_k) = w_k . torque
      const float gtx = acc.gx + 2.f * p.gravity * tx;
      const float gty = acc.gy + 2.f * p.gravity * ty;
      const float gtz = acc.gz + 2.f * p.gravity * tz;
      const float gphi = acc.t[2];
      const float gpsi = -sphi * acc.t[0] + cphi * acc.t[1];
      const float gth = -(cphi * spsi * acc.t[0] + sphi * spsi * acc.t[1] + cpsi * acc.t[2]);
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
      // ---- fused ADAM step on lanes 0..5 (optax.adam form) ----
      const bool ok = isfinite(gtx) & isfinite(gty) & isfinite(gtz) & isfinite(gphi) & isfinite(gpsi) &
                      isfinite(gth);
      if (!ok) {
        status |= ATT_STATUS_NONFINITE_GRAD;
      } else if (tl < 6) {
        const float t = (float)(p.step0 + s + 1);
        my_m = fmaf(p.b1, my_m, (1.f - p.b1) * gk);
        my_v = fmaf(p.b2, my_v, (1.f - p.b2) * gk * gk);
        const float mh = my_m / (1.f - powf(p.b1, t));
        const float vh = my_v / (1.f - powf(p.b2, t));
        const float lr = (tl < 3) ? p.lr_rot : p.lr_trans;
        my_x -= lr * mh / (sqrtf(vh) + p.eps);
      }
    }

    if (MODE == MODE_MIN && valid) {
      if (tl < 6) {
        p.pose_out[(long long)b * 6 + tl] = my_x;
        if (p.adam != nullptr) {
          p.adam[(long long)b * 12 + tl] = my_m;
          p.adam[(long long)b * 12 + 6 + tl] = my_v;
        }
      }
    }
    if ((MODE == MODE_MIN || MODE == MODE_EVAL) && valid && tl == 0 && p.status != nullptr) p.status[b] = status;

    if (p.counter != nullptr) {
      int t0 = 0;
      if (lane == 0) t0 = atomicAdd(p.counter, 1);
      tile = __shfl_sync(0xffffffffu, t0, 0);
    } else {
      tile += nwarps;
    }
  }

  if (MODE == MODE_MIN && p.stats != nullptr) {
    unsigned long long v[3] = {c_grid, c_look, c_ent};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
      if (lane == 0 && v[k]) atomicAdd(p.stats + k, v[k]);
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int MODE>
static cudaError_t launch_mode(const KParams& p, int S, int blocks, int threads, cudaStream_t st) {
  switch (S) {
    case 8: score_kernel<8, MODE><<<blocks, threads, 0, st>>>(p); break;
    case 16: score_kernel<16, MODE><<<blocks, threads, 0, st>>>(p); break;
    case 32: score_kernel<32, MODE><<<blocks, threads, 0, st>>>(p); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int MODE>
static const void* kernel_ptr(int S) {
  switch (S) {
    case 8: return (const void*)score_kernel<8, MODE>;
    case 16: return (const void*)score_kernel<16, MODE>;
    case 32: return (const void*)score_kernel<32, MODE>;
  }
  return nullptr;
}

cudaError_t launch_score(const KParams& p, int mode, int S, int blocks, int threads, cudaStream_t st) {
  switch (mode) {
    case MODE_EVAL: return launch_mode<MODE_EVAL>(p, S, blocks, threads, st);
    case MODE_EVAL_MAT: return launch_mode<MODE_EVAL_MAT>(p, S, blocks, threads, st);
    case MODE_MIN: return launch_mode<MODE_MIN>(p, S, blocks, threads, st);
    case MODE_BWD: return launch_mode<MODE_BWD>(p, S, blocks, threads, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t occupancy_blocks(int mode, int S, int threads, int* blocks_per_sm) {
  const void* k = nullptr;
  switch (mode) {
    case MODE_EVAL: k = kernel_ptr<MODE_EVAL>(S); break;
    case MODE_EVAL_MAT: k = kernel_ptr<MODE_EVAL_MAT>(S); break;
    case MODE_MIN: k = kernel_ptr<MODE_MIN>(S); break;
    case MODE_BWD: k = kernel_ptr<MODE_BWD>(S); break;
  }
  if (k == nullptr) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, 0);
}

}  // namespace att
