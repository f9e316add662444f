// Explicit all-pairs ATTRACT energy (and pose gradient): every ligand bead
// against every receptor bead, no grid -- the rescoring path of the reference,
// test-energy.py:46-58 (delta over all pairs, nonbon of every d^2, summed per
// structure), with ATTRACT's --rcut as an optional distance cutoff.
//
// One block of 8 warps per pose (grid-stride over poses).  The receptor streams
// through shared memory in tiles of AP_TILE beads; a warp takes one ligand bead
// at a time against 32 consecutive receptor beads per step (conflict-free
// 16-byte shared loads).  The pair-parameter row depends on the receptor type:
// a lane keeps the last row it loaded and reloads only when the type changes,
// so a receptor sorted by type (the host wrapper sorts it) reads each row once
// per run of equal types instead of once per pair.  Per bead, the warp's lane
// sums (energy and force, float) are reduced with shuffles and added to the
// bead's accumulator in shared memory (double); the torque -- or x (x) g for the
// 4x4 form -- is formed once per bead from its total force, and the block sums
// the beads in double.
#include <math.h>

#include "common.cuh"

namespace att {
int report_error(int code, const char* msg);

constexpr int AP_THREADS = 256;
constexpr int AP_WARPS = AP_THREADS / 32;
constexpr int AP_TILE = 2048;   // receptor beads per shared-memory tile (32 KB)
constexpr int AP_BEADS = 512;   // ligand beads per pass (their accumulators: 16 KB)
constexpr size_t AP_SMEM = (size_t)AP_TILE * sizeof(float4) + (size_t)AP_BEADS * 4 * sizeof(double) +
                           (size_t)AP_WARPS * 13 * sizeof(double);

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
      for (int w = 0; w < AP_WARPS; ++w) s += red[w * NV + k];
      v[k] = s;
    }
  }
  __syncthreads();
}

// 1/d2: the approximate reciprocal refined by one Newton step (within 1 ulp)
__device__ __forceinline__ float recip_nr(float d2) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d2));
  return r * fmaf(-d2, r, 2.f);
}

__global__ void __launch_bounds__(AP_THREADS) allpairs_kernel(const __grid_constant__ AllPairsParams p) {
  extern __shared__ __align__(16) unsigned char ap_smem[];
  float4* s_rec = reinterpret_cast<float4*>(ap_smem);
  double* s_acc = reinterpret_cast<double*>(ap_smem + (size_t)AP_TILE * sizeof(float4));  // [AP_BEADS][4]
  double* red = s_acc + AP_BEADS * 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
    // energy, force and the lever-arm sums (torque, or x (x) g for the 4x4 form)
    double acc[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) acc[k] = 0.0;
    for (int i0 = 0; i0 < p.n_lig; i0 += AP_BEADS) {
      const int nb = min(AP_BEADS, p.n_lig - i0);
      for (int k = threadIdx.x; k < nb * 4; k += AP_THREADS) s_acc[k] = 0.0;
      for (int j0 = 0; j0 < p.n_rec; j0 += AP_TILE) {
        const int nt = min(AP_TILE, p.n_rec - j0);
        __syncthreads();  // the previous tile has been read
        for (int j = threadIdx.x; j < nt; j += AP_THREADS) s_rec[j] = __ldg(p.rec + j0 + j);
        __syncthreads();
        for (int i = i0 + warp; i < i0 + nb; i += AP_WARPS) {  // warp-uniform
          const float4 x = __ldg(p.lig + i);
          const int lt = __float_as_int(x.w);
          if ((unsigned)lt >= (unsigned)p.n_ltypes) continue;  // no pair table row: contributes nothing
          const float X = fmaf(x.x, m[0], fmaf(x.y, m[3], fmaf(x.z, m[6], t[0])));
          const float Y = fmaf(x.x, m[1], fmaf(x.y, m[4], fmaf(x.z, m[7], t[1])));
          const float Z = fmaf(x.x, m[2], fmaf(x.y, m[5], fmaf(x.z, m[8], t[2])));
          const float4* prow = p.pair + (size_t)lt * p.n_rtypes * 2;
          float e = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
          int cur = -1;
          float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;  // rc, ac, emin, rmin2 / ivor, eplat, -, rcap2
          for (int j = lane; j < nt; j += 32) {
            const float4 r = s_rec[j];
            const int rt = __float_as_int(r.w);
            const float dx = X - r.x, dy = Y - r.y, dz = Z - r.z;
            const float dsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool hit = ((unsigned)rt < (unsigned)p.n_rtypes) & ((p.rcut2 <= 0.f) | (dsq < p.rcut2));
            const int rtc = hit ? rt : 0;
            if (rtc != cur) {  // a new receptor type: its row
              ldg_f4x2(prow + rtc * 2, p0, p1);
              cur = rtc;
            }
            const float d2 = fmaxf(dsq, p1.w);
            const float rr2 = recip_nr(d2);
            const float rr6 = rr2 * rr2 * rr2;
            const float vlj = fmaf(p0.x, rr2, -p0.y) * rr6;
            const bool near = d2 < p0.w;
            const float en = near ? fmaf(p1.x - 1.f, p0.z, vlj) : p1.x * vlj;
            float gm2 = rr6 * rr2 * fmaf(-8.f * p0.x, rr2, 6.f * p0.y);  // 2 dnonbon/d(d^2)
            gm2 = near ? gm2 : p1.x * gm2;
            gm2 = (dsq < p1.w) ? 0.f : gm2;
            const float gf = hit ? gm2 : 0.f;
            e += hit ? en - p1.y : 0.f;
            gx = fmaf(gf, dx, gx);
            gy = fmaf(gf, dy, gy);
            gz = fmaf(gf, dz, gz);
          }
#pragma unroll
          for (int off = 16; off >= 1; off >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, off);
            gx += __shfl_xor_sync(0xffffffffu, gx, off);
            gy += __shfl_xor_sync(0xffffffffu, gy, off);
            gz += __shfl_xor_sync(0xffffffffu, gz, off);
          }
          if (lane == 0) {  // bead i belongs to this warp alone
            double* a = s_acc + (i - i0) * 4;
            a[0] += e;
            a[1] += gx;
            a[2] += gy;
            a[3] += gz;
          }
        }
      }
      __syncthreads();  // every warp's accumulators written (or just cleared)
      // per bead of this pass: energy, force and its lever-arm terms
      for (int i = i0 + threadIdx.x; i < i0 + nb; i += AP_THREADS) {
        const double* a = s_acc + (i - i0) * 4;
        const double e = a[0], gx = a[1], gy = a[2], gz = a[3];
        const float4 x = __ldg(p.lig + i);
        acc[0] += e;
        acc[1] += gx;
        acc[2] += gy;
        acc[3] += gz;
        if (mat) {  // dE/dM[r][c] = sum_i x_r g_c
          const double xr[3] = {x.x, x.y, x.z}, gc[3] = {gx, gy, gz};
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[4 + r * 3 + c] += xr[r] * gc[c];
        } else {  // torque about the pose centre: (X - t) x g, X - t = x M
          const double ax = fmaf(x.x, m[0], fmaf(x.y, m[3], x.z * m[6]));
          const double ay = fmaf(x.x, m[1], fmaf(x.y, m[4], x.z * m[7]));
          const double az = fmaf(x.x, m[2], fmaf(x.y, m[5], x.z * m[8]));
          acc[4] += ay * gz - az * gy;
          acc[5] += az * gx - ax * gz;
          acc[6] += ax * gy - ay * gx;
        }
      }
      __syncthreads();  // the accumulators are read before the next pass clears them
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
  cudaError_t e = cudaFuncSetAttribute(allpairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)AP_SMEM);
  if (e != cudaSuccess) return report_error(ATT_E_CUDA, cudaGetErrorString(e));
  int per_sm = 1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, allpairs_kernel, AP_THREADS, AP_SMEM);
  if (e != cudaSuccess) return report_error(ATT_E_CUDA, cudaGetErrorString(e));
  const int blocks = (int)min((long long)n_poses, (long long)sms * max(per_sm, 1));
  allpairs_kernel<<<blocks, AP_THREADS, AP_SMEM, (cudaStream_t)stream>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report_error(ATT_E_CUDA, cudaGetErrorString(e));
  return ATT_OK;
}
