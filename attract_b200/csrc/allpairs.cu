// Explicit all-pairs ATTRACT energy (and pose gradient): every ligand bead
// against every receptor bead, no grid -- the rescoring path of the reference,
// test-energy.py:46-58 (delta over all pairs, nonbon of every d^2, summed per
// structure), with ATTRACT's --rcut as an optional distance cutoff.
//
// One block per pose (grid-stride over poses).  The receptor streams through
// shared memory in tiles of ALLPAIRS_TILE beads.  A thread holds one ligand
// bead in registers and takes a slice of every tile: with n ligand beads,
// 256 / n threads share each bead (a small ligand still fills the block), so
// a warp reads at most a few receptor beads at a time (broadcasts).  Per-thread
// sums (energy in float, force, lever-arm products) are reduced over the block
// in double; the torque is linear in the force, so partial forces of one bead
// add up correctly.
#include <math.h>

#include "common.cuh"

namespace att {
int report_error(int code, const char* msg);

constexpr int ALLPAIRS_THREADS = 256;
constexpr int ALLPAIRS_TILE = 1024;  // receptor beads per shared-memory tile (16 KB)

struct AllPairsParams {
  const float4* rec;   // [n_rec] x, y, z, receptor type (int bits)
  const float4* lig;   // [n_lig] x, y, z, ligand type (int bits)
  const float* pose;   // [B][6] Euler + translation, or [B][16] row-vector 4x4
  const float4* pair;  // [n_ltypes][n_rtypes][2]: rc, ac, emin, rmin2 / ivor, eplat, -, rcap2
  float* energy;       // [B]
  float* grad;         // [B][6] or [B][16], may be NULL
  float rcut2;         // <= 0: no cutoff
  int n_rec, n_lig, n_poses, pose_format, n_rtypes, n_ltypes;
};

// block-wide double sum of v[0..n); result valid in thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[warp * NV + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < ALLPAIRS_THREADS / 32; ++w) s += red[w * NV + k];
      v[k] = s;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(ALLPAIRS_THREADS) allpairs_kernel(const __grid_constant__ AllPairsParams p) {
  __shared__ float4 s_rec[ALLPAIRS_TILE];
  __shared__ double red[(ALLPAIRS_THREADS / 32) * 13];
  const bool mat = p.pose_format == 1;
  for (int b = blockIdx.x; b < p.n_poses; b += gridDim.x) {
    // pose -> row-vector rotation M (X = x M + t) and, for Euler poses, the angles
    float m[9], t[3], sphi = 0.f, cphi = 1.f, spsi = 0.f, cpsi = 1.f;
    if (mat) {
      const float* P = p.pose + (long long)b * 16;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) m[r * 3 + c] = __ldg(P + r * 4 + c);
#pragma unroll
      for (int c = 0; c < 3; ++c) t[c] = __ldg(P + 12 + c);
    } else {
      const float* P = p.pose + (long long)b * 6;
      float sth, cth;
      sincosf(__ldg(P + 0), &sphi, &cphi);
      sincosf(__ldg(P + 1), &spsi, &cpsi);
      sincosf(__ldg(P + 2), &sth, &cth);
      // column-form Q = Rz(phi) Ry(psi) Rz(-theta); the row-vector M is its transpose
      const float q00 = cphi * cpsi * cth + sphi * sth, q01 = cphi * cpsi * sth - sphi * cth, q02 = cphi * spsi;
      const float q10 = sphi * cpsi * cth - cphi * sth, q11 = sphi * cpsi * sth + cphi * cth, q12 = sphi * spsi;
      const float q20 = -spsi * cth, q21 = -spsi * sth, q22 = cpsi;
      m[0] = q00; m[1] = q10; m[2] = q20;
      m[3] = q01; m[4] = q11; m[5] = q21;
      m[6] = q02; m[7] = q12; m[8] = q22;
#pragma unroll
      for (int c = 0; c < 3; ++c) t[c] = __ldg(P + 3 + c);
    }
    // per thread: energy, force, and the lever-arm sums (torque, or x (x) g for the 4x4 form)
    double acc[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) acc[k] = 0.0;
    // threads per bead (receptor slices) and this thread's bead / slice
    const int nsl = p.n_lig < ALLPAIRS_THREADS ? ALLPAIRS_THREADS / p.n_lig : 1;
    const int per = ALLPAIRS_THREADS / nsl;  // beads per pass
    const int sl = (int)threadIdx.x / per;
    for (int i0 = 0; i0 < p.n_lig; i0 += per) {
      const int i = i0 + (int)threadIdx.x % per;
      const bool live = i < p.n_lig && sl < nsl;
      float4 x = live ? __ldg(p.lig + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      const int lt = live ? __float_as_int(x.w) : -1;
      const float X = fmaf(x.x, m[0], fmaf(x.y, m[3], fmaf(x.z, m[6], t[0])));
      const float Y = fmaf(x.x, m[1], fmaf(x.y, m[4], fmaf(x.z, m[7], t[1])));
      const float Z = fmaf(x.x, m[2], fmaf(x.y, m[5], fmaf(x.z, m[8], t[2])));
      const bool lok = live && (unsigned)lt < (unsigned)p.n_ltypes;
      const float4* prow = p.pair + (long long)(lok ? lt : 0) * p.n_rtypes * 2;
      float e = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
      for (int j0 = 0; j0 < p.n_rec; j0 += ALLPAIRS_TILE) {
        const int nt = min(ALLPAIRS_TILE, p.n_rec - j0);
        __syncthreads();  // the previous tile has been read
        for (int j = threadIdx.x; j < nt; j += ALLPAIRS_THREADS) s_rec[j] = __ldg(p.rec + j0 + j);
        __syncthreads();
        if (lok) {
          for (int j = sl; j < nt; j += nsl) {
            const float4 r = s_rec[j];
            const int rt = __float_as_int(r.w);
            const float dx = X - r.x, dy = Y - r.y, dz = Z - r.z;
            const float dsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool hit = ((unsigned)rt < (unsigned)p.n_rtypes) & ((p.rcut2 <= 0.f) | (dsq < p.rcut2));
            float4 p0, p1;  // rc, ac, emin, rmin2 / ivor, eplat, -, rcap2
            ldg_f4x2(prow + (hit ? rt : 0) * 2, p0, p1);
            const float d2 = fmaxf(dsq, p1.w);
            const float rr2 = 1.0f / d2;
            const float rr6 = rr2 * rr2 * rr2;
            const float vlj = fmaf(p0.x, rr2, -p0.y) * rr6;
            const bool near = d2 < p0.w;
            const float en = near ? fmaf(p1.x - 1.f, p0.z, vlj) : p1.x * vlj;
            float gm = rr6 * rr2 * fmaf(-4.f * p0.x, rr2, 3.f * p0.y);
            gm = near ? gm : p1.x * gm;
            gm = (dsq < p1.w) ? 0.f : gm;
            const float gf = hit ? 2.f * gm : 0.f;
            e += hit ? en - p1.y : 0.f;
            gx = fmaf(gf, dx, gx);
            gy = fmaf(gf, dy, gy);
            gz = fmaf(gf, dz, gz);
          }
        }
      }
      acc[0] += e;
      acc[1] += gx;
      acc[2] += gy;
      acc[3] += gz;
      if (mat) {  // dE/dM[r][c] = sum_i x_r g_c
        const float xr[3] = {x.x, x.y, x.z}, gc[3] = {gx, gy, gz};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[4 + r * 3 + c] += (double)xr[r] * gc[c];
      } else {  // torque about the pose centre: (X - t) x g
        const float ax = X - t[0], ay = Y - t[1], az = Z - t[2];
        acc[4] += (double)ay * gz - (double)az * gy;
        acc[5] += (double)az * gx - (double)ax * gz;
        acc[6] += (double)ax * gy - (double)ay * gx;
      }
    }
    block_sum<13>(acc, red);
    if (threadIdx.x == 0) {
      p.energy[b] = (float)acc[0];
      if (p.grad != nullptr) {
        if (mat) {
          float* g = p.grad + (long long)b * 16;
#pragma unroll
          for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) g[r * 4 + c] = (float)acc[4 + r * 3 + c];
            g[r * 4 + 3] = 0.f;
          }
          g[12] = (float)acc[1]; g[13] = (float)acc[2]; g[14] = (float)acc[3]; g[15] = 0.f;
        } else {
          // dE/d(angle_k) = w_k . torque with w_phi = (0,0,1), w_psi = (-sin phi, cos phi, 0),
          // w_theta = -(cos phi sin psi, sin phi sin psi, cos psi)
          float* g = p.grad + (long long)b * 6;
          const double tx = acc[4], ty = acc[5], tz = acc[6];
          g[0] = (float)tz;
          g[1] = (float)(-sphi * tx + cphi * ty);
          g[2] = (float)(-(cphi * spsi * tx + sphi * spsi * ty + cpsi * tz));
          g[3] = (float)acc[1]; g[4] = (float)acc[2]; g[5] = (float)acc[3];
        }
      }
    }
  }
}

}  // namespace att

using namespace att;

extern "C" int att_allpairs_energy(const float* rec_dev, int n_rec, const float* lig_dev, int n_lig,
                                   const float* pose_dev, int n_poses, int pose_format, const float* pair_dev,
                                   int n_rtypes, int n_ltypes, float rcut, float* energy_dev, float* grad_dev,
                                   void* stream) {
  auto bad = [](const char* m) { return report_error(ATT_E_INVALID, m); };
  auto al16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  if (n_rec < 0 || n_lig < 1 || n_poses < 0) return bad("att_allpairs_energy: n_rec >= 0, n_lig >= 1, n_poses >= 0");
  if (n_rtypes < 1 || n_ltypes < 1) return bad("att_allpairs_energy: empty pair table");
  if (pose_format != 0 && pose_format != 1) return bad("att_allpairs_energy: pose_format must be 0 or 1");
  if ((n_rec && !rec_dev) || !lig_dev || !pair_dev || (n_poses && (!pose_dev || !energy_dev)))
    return bad("att_allpairs_energy: NULL buffer");
  if ((rec_dev && !al16(rec_dev)) || !al16(lig_dev) || (reinterpret_cast<uintptr_t>(pair_dev) & 31u))
    return bad("att_allpairs_energy: receptor and ligand must be 16-byte, the pair table 32-byte aligned");
  if (!(rcut >= 0.f)) return bad("att_allpairs_energy: rcut must be >= 0 (0 = no cutoff)");
  if (n_poses == 0) return ATT_OK;
  AllPairsParams p;
  p.rec = reinterpret_cast<const float4*>(rec_dev);
  p.lig = reinterpret_cast<const float4*>(lig_dev);
  p.pose = pose_dev;
  p.pair = reinterpret_cast<const float4*>(pair_dev);
  p.energy = energy_dev;
  p.grad = grad_dev;
  p.rcut2 = rcut > 0.f ? rcut * rcut : 0.f;
  p.n_rec = n_rec;
  p.n_lig = n_lig;
  p.n_poses = n_poses;
  p.pose_format = pose_format;
  p.n_rtypes = n_rtypes;
  p.n_ltypes = n_ltypes;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = (int)min((long long)n_poses, (long long)sms * 8);
  allpairs_kernel<<<blocks, ALLPAIRS_THREADS, 0, (cudaStream_t)stream>>>(p);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return report_error(ATT_E_CUDA, cudaGetErrorString(e));
  return ATT_OK;
}
