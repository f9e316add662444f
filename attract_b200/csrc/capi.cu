// The extern "C" boundary: argument validation, device views, launches.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "common.cuh"

namespace att {
cudaError_t launch_score(const KParams& p, int mode, int S, int K, int blocks, int threads, cudaStream_t st);
cudaError_t occupancy_blocks(int mode, int S, int K, int threads, int rec_slot, int* blocks_per_sm);
cudaError_t kernel_status(int* out, int clear, cudaStream_t st);
cudaError_t kernel_debug_info(unsigned long long* out3, int clear, cudaStream_t st);
int beads_per_lane(int S, int max_beads);
size_t score_smem_bytes(int K, int threads, int rec_slot);
cudaError_t launch_build_potential(const AttGridGeom& g, const float* rec, int n_rec, const float* pair,
                                   int n_rtypes, int n_ltypes, float cutoff, int outer, float* out,
                                   cudaStream_t st);
long long nb_workspace_bytes(long long nvox);
cudaError_t launch_nb_count(const AttGridGeom& g, const float* rec, int n_rec, float radius, uint32_t* hdr,
                            unsigned long long* total, void* ws, cudaStream_t st);
cudaError_t launch_nb_fill(const AttGridGeom& g, const float* rec, int n_rec, float radius, const uint32_t* hdr,
                           uint16_t* list, cudaStream_t st);
cudaError_t launch_repack(const AttGridGeom& g, const float* inner, const float* outer, void* bricks,
                          cudaStream_t st);
cudaError_t launch_nb_pack(const uint32_t* hdr, const uint16_t* list, long long nvox, int rec_bytes, void* out,
                           cudaStream_t st);
}  // namespace att

using namespace att;

static thread_local char g_err[512] = "";

static int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

namespace att {
// error reporting for entry points defined in other translation units
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace att

static int cuda_fail(cudaError_t e, const char* where) {
  return fail(ATT_E_CUDA, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define REQUIRE(cond, ...)                          \
  do {                                              \
    if (!(cond)) return fail(ATT_E_INVALID, __VA_ARGS__); \
  } while (0)

extern "C" const char* att_last_error_string(void) { return g_err; }
extern "C" const char* att_version(void) { return "attract_b200 0.1 (sm_100a)"; }

static bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// dynamic shared memory per block of the scoring kernels: 227 KB less the
// static grid-descriptor copies (ATT_MAX_GRIDS KGrid) and slack
static const size_t kDynSmemLimit = 227 * 1024 - 4096;

namespace att {
// geometry validation shared by every entry point that takes an AttGridGeom
int check_geom(const AttGridGeom* g) {
  REQUIRE(g != nullptr, "geometry is NULL");
  for (int k = 0; k < 3; ++k) {
    REQUIRE(g->dim[k] >= 2, "dim[%d] = %d must be >= 2", k, g->dim[k]);
    REQUIRE(g->dim2[k] >= 0, "dim2[%d] = %d must be >= 0", k, g->dim2[k]);
  }
  REQUIRE(g->spacing > 0.f, "spacing must be > 0");
  REQUIRE(g->plateau >= 0.f, "plateau must be >= 0");
  REQUIRE(g->n_types >= 1 && g->n_types <= 65535, "n_types = %d out of range", g->n_types);
  return ATT_OK;
}
}  // namespace att

long long att_grid_brick_bytes(const AttGridGeom* g, int with_outer) {
  if (check_geom(g) != ATT_OK) return -1;
  const long long ni = (long long)(g->dim[0] - 1) * (g->dim[1] - 1) * (g->dim[2] - 1);
  long long no = 0;
  if (with_outer && g->dim2[0] >= 2 && g->dim2[1] >= 2 && g->dim2[2] >= 2)
    no = (long long)(g->dim2[0] - 1) * (g->dim2[1] - 1) * (g->dim2[2] - 1);
  return (long long)g->n_types * (ni + no) * 128;
}

static int make_kgrid(const AttGrid* a, int gi, KGrid* k) {
  int rc = check_geom(&a->geom);
  if (rc) return rc;
  const AttGridGeom& g = a->geom;
  const long long ni = (long long)(g.dim[0] - 1) * (g.dim[1] - 1) * (g.dim[2] - 1);
  REQUIRE(a->pair != nullptr, "grid %d: pair table is NULL", gi);
  REQUIRE(a->n_rtypes >= 1 && a->n_ltypes >= 1, "grid %d: n_rtypes/n_ltypes must be >= 1", gi);
  REQUIRE(a->n_rec >= 0 && a->n_rec < (int)ATT_NB_EMPTY, "grid %d: n_rec = %d out of range [0, 65535)", gi,
          a->n_rec);
  REQUIRE(a->n_rec == 0 || (a->rec != nullptr && aligned(a->rec, 16)), "grid %d: rec NULL or not 16-B aligned", gi);
  REQUIRE(aligned(a->pair, 32), "grid %d: pair table not 32-B aligned", gi);
  if (a->bricks != nullptr) {
    REQUIRE(aligned(a->bricks, 128), "grid %d: bricks must be 128-B aligned", gi);
    REQUIRE(a->n_inner_bricks == ni, "grid %d: n_inner_bricks = %lld, expected %lld", gi, a->n_inner_bricks, ni);
    if (a->n_outer_bricks != 0) {
      REQUIRE(g.dim2[0] >= 2 && g.dim2[1] >= 2 && g.dim2[2] >= 2, "grid %d: outer bricks need dim2 >= 2", gi);
      const long long no = (long long)(g.dim2[0] - 1) * (g.dim2[1] - 1) * (g.dim2[2] - 1);
      REQUIRE(a->n_outer_bricks == no, "grid %d: n_outer_bricks = %lld, expected %lld", gi, a->n_outer_bricks, no);
    }
  }
  if (a->nb_hdr != nullptr) {
    REQUIRE(aligned(a->nb_hdr, 8), "grid %d: nb_hdr not 8-B aligned", gi);
    REQUIRE(a->n_nb_entries == 0 || a->nb_list != nullptr, "grid %d: nb_list is NULL", gi);
    REQUIRE(a->nb_rec != nullptr && aligned(a->nb_rec, 16), "grid %d: nb_rec NULL or not 16-B aligned", gi);
    REQUIRE(a->nb_rec_bytes == 32 || a->nb_rec_bytes == 64 || a->nb_rec_bytes == 128,
            "grid %d: nb_rec_bytes = %d (32, 64 or 128)", gi, a->nb_rec_bytes);
    REQUIRE(a->nb_refine >= 0 && a->nb_refine <= 4 && a->nb_refine != 3, "grid %d: nb_refine = %d (0, 1, 2 or 4)",
            gi, a->nb_refine);
  }
  memset(k, 0, sizeof(*k));
  k->ox = g.origin[0];
  k->oy = g.origin[1];
  k->oz = g.origin[2];
  k->inv_s = 1.f / g.spacing;
  k->fdx1 = (float)(g.dim[0] - 1);
  k->fdy1 = (float)(g.dim[1] - 1);
  k->fdz1 = (float)(g.dim[2] - 1);
  k->fex1 = (float)(g.dim2[0] - 1);
  k->fey1 = (float)(g.dim2[1] - 1);
  k->fez1 = (float)(g.dim2[2] - 1);
  k->ext = (float)g.extension;
  k->plateau = g.plateau;
  k->plateau2 = g.plateau * g.plateau;
  k->plateau_x2 = 2.f * g.plateau;
  k->dx = g.dim[0];
  k->dy = g.dim[1];
  k->dz = g.dim[2];
  k->dx2 = g.dim2[0];
  k->dy2 = g.dim2[1];
  k->dz2 = g.dim2[2];
  k->n_types = g.n_types;
  k->n_rec = a->n_rec;
  k->n_rtypes = a->n_rtypes;
  k->n_ltypes = a->n_ltypes;
  k->has_outer = (a->bricks != nullptr && a->n_outer_bricks > 0) ? 1 : 0;
  k->type_stride = ni + (k->has_outer ? a->n_outer_bricks : 0);
  k->n_inner = ni;
  k->n_list = a->n_nb_entries;
  const int rf = a->nb_refine > 1 ? a->nb_refine : 1;  // list grid = inner grid refined rf times
  k->nb_scale = (float)rf;
  k->ndy = (g.dim[1] - 1) * rf + 1;
  k->ndz = (g.dim[2] - 1) * rf + 1;
  k->n_vox = (long long)((g.dim[0] - 1) * rf + 1) * k->ndy * k->ndz;
  k->n_bricks = (long long)g.n_types * k->type_stride;
  k->bricks = reinterpret_cast<const float4*>(a->bricks);
  k->nb_hdr = reinterpret_cast<const uint2*>(a->nb_hdr);
  k->nb_list = a->nb_list;
  if (a->nb_hdr != nullptr) {
    k->nb_rec = reinterpret_cast<const unsigned char*>(a->nb_rec);
    k->nb_rec_bytes = a->nb_rec_bytes;
    k->nb_inline = ATT_NB_INLINE(a->nb_rec_bytes);
  }
  k->rec = reinterpret_cast<const float4*>(a->rec);
  k->pair = reinterpret_cast<const float4*>(a->pair);
  // the scoring kernels remember which brick and which list point a bead's
  // shared-memory slots hold as 32-bit indices
  REQUIRE(k->n_bricks <= 2147483647LL, "grid %d: %lld bricks; at most 2^31 - 1", gi, k->n_bricks);
  REQUIRE(a->nb_hdr == nullptr || k->n_vox <= 2147483647LL, "grid %d: %lld list points; at most 2^31 - 1", gi,
          k->n_vox);
  return ATT_OK;
}

static int fill_common(KParams* p, const AttGrid* grids, int n_grids, const AttLigands* ligs,
                       const AttSegment* segs, int n_segs, const int* seg_tile, int n_tiles, int n_pose_rows,
                       const float* pose,
                       const int* pose_lig, const AttEvalCfg* cfg, const AttLaunchCfg* launch, int* S, int* K,
                       int* threads) {
  REQUIRE(grids != nullptr && n_grids >= 1 && n_grids <= ATT_MAX_GRIDS, "n_grids = %d out of range [1, %d]",
          n_grids, ATT_MAX_GRIDS);
  REQUIRE(ligs != nullptr && ligs->beads != nullptr && ligs->offset != nullptr && ligs->n_lig >= 1,
          "ligands: beads/offset NULL or n_lig < 1");
  REQUIRE(aligned(ligs->beads, 16), "ligand beads not 16-B aligned");
  REQUIRE(segs != nullptr && n_segs >= 1 && seg_tile != nullptr, "segments / seg_tile missing");
  REQUIRE(n_tiles >= 0, "n_tiles < 0");
  REQUIRE(n_pose_rows >= 0, "n_pose_rows < 0");
  REQUIRE(pose != nullptr || n_tiles == 0, "pose is NULL");
  REQUIRE(cfg != nullptr, "eval cfg is NULL");
  REQUIRE(cfg->grad_mode == ATT_GRAD_REFERENCE || cfg->grad_mode == ATT_GRAD_ANALYTIC, "grad_mode %d unknown",
          cfg->grad_mode);
  int s = (launch && launch->lanes_per_pose) ? launch->lanes_per_pose : 8;
  REQUIRE(s == 8 || s == 16 || s == 32, "lanes_per_pose = %d (8, 16 or 32)", s);
  *S = s;
  REQUIRE(ligs->max_beads >= 1, "ligands: max_beads = %d", ligs->max_beads);
  REQUIRE(ligs->n_beads >= ligs->max_beads, "ligands: n_beads = %d < max_beads = %d", ligs->n_beads,
          ligs->max_beads);
  *K = beads_per_lane(s, ligs->max_beads);
  int t = (launch && launch->block_threads) ? launch->block_threads : 128;
  REQUIRE(t == 32 || t == 64 || t == 96 || t == 128, "block_threads = %d (32, 64, 96 or 128)", t);
  *threads = t;
  memset(p, 0, sizeof(*p));
  int rec_slot = 0;  // neighbour-record slot: the largest record of any grid
  for (int i = 0; i < n_grids; ++i) {
    int rc = make_kgrid(&grids[i], i, &p->grid[i]);
    if (rc) return rc;
    if (p->grid[i].nb_rec_bytes > rec_slot) rec_slot = p->grid[i].nb_rec_bytes;
  }
  p->rec_slot = rec_slot;
  REQUIRE(!launch || launch->test_flags == 0, "AttLaunchCfg.test_flags is reserved and must be 0");
  p->test_flags = 0;
  if (!(launch && launch->block_threads)) {  // default: the largest block whose shared memory fits
    while (t > 32 && score_smem_bytes(*K, t, rec_slot) > kDynSmemLimit) t -= 32;
    *threads = t;
  }
  REQUIRE(score_smem_bytes(*K, t, rec_slot) <= kDynSmemLimit,
          "%d threads x %d beads per lane need %zu B of shared memory", t, *K, score_smem_bytes(*K, t, rec_slot));
  p->lig_beads = reinterpret_cast<const float4*>(ligs->beads);
  p->lig_off = ligs->offset;
  p->segs = segs;
  p->seg_tile = seg_tile;
  p->n_segs = n_segs;
  p->n_tiles = n_tiles;
  p->n_grids = n_grids;
  p->n_lig = ligs->n_lig;
  p->max_beads = ligs->max_beads;
  p->n_lig_beads = ligs->n_beads;
  p->n_pose_rows = n_pose_rows;
  p->pose_in = pose;
  p->pose_lig = pose_lig;
  p->grad_mode = cfg->grad_mode;
  p->quirk = (cfg->flags & ATT_FLAG_TRILINEAR_QUIRK) ? 1 : 0;
  p->gravity = cfg->gravity;
  return ATT_OK;
}

extern "C" int att_energrad(const AttGrid* grids, int n_grids, const AttLigands* ligs, const AttSegment* segs_dev,
                            int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows, const float* pose_dev,
                            const int* pose_lig_dev, const AttEvalCfg* cfg, float* energy_dev, float* grad_dev,
                            int* status_dev, const AttLaunchCfg* launch, void* stream) {
  KParams p;
  int S = 8, K = 1, threads = 128;
  int rc = fill_common(&p, grids, n_grids, ligs, segs_dev, n_segs, seg_tile_dev, n_tiles, n_pose_rows, pose_dev, pose_lig_dev,
                       cfg, launch, &S, &K, &threads);
  if (rc) return rc;
  REQUIRE(energy_dev != nullptr || n_tiles == 0, "energy output is NULL");
  REQUIRE(cfg->pose_format == 0 || cfg->pose_format == 1, "pose_format %d unknown", cfg->pose_format);
  p.energy = energy_dev;
  p.grad = grad_dev;
  p.status = status_dev;
  if (n_tiles == 0) return ATT_OK;
  const int wpb = threads / 32;
  const int blocks = (n_tiles + wpb - 1) / wpb;
  cudaError_t e = launch_score(p, cfg->pose_format == 1 ? MODE_EVAL_MAT : MODE_EVAL, S, K, blocks, threads,
                               (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_energrad launch");
  return ATT_OK;
}

static int persistent_blocks(int mode, int S, int K, int threads, int rec_slot, const AttLaunchCfg* launch, int n_tiles,
                             int* blocks) {
  if (launch && launch->blocks > 0) {
    *blocks = launch->blocks;
    return ATT_OK;
  }
  int dev = 0, sms = 0, per = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = occupancy_blocks(mode, S, K, threads, rec_slot, &per);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
  if (per < 1) per = 1;
  const int wpb = threads / 32;
  int b = sms * per;
  const int need = (n_tiles + wpb - 1) / wpb;
  if (b > need) b = need;
  if (b < 1) b = 1;
  *blocks = b;
  return ATT_OK;
}

extern "C" int att_minimise(const AttGrid* grids, int n_grids, const AttLigands* ligs, const AttSegment* segs_dev,
                            int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows, const float* pose_in_dev,
                            float* pose_out_dev, const int* pose_lig_dev, float* adam_state_dev,
                            const AttAdamCfg* cfg, int steps, float* energy_dev, int* status_dev,
                            int* work_counter_dev, unsigned long long* stats_dev, const AttLaunchCfg* launch,
                            void* stream) {
  REQUIRE(cfg != nullptr, "adam cfg is NULL");
  KParams p;
  int S = 8, K = 1, threads = 128;
  int rc = fill_common(&p, grids, n_grids, ligs, segs_dev, n_segs, seg_tile_dev, n_tiles, n_pose_rows, pose_in_dev,
                       pose_lig_dev, &cfg->eval, launch, &S, &K, &threads);
  if (rc) return rc;
  REQUIRE(cfg->eval.pose_format == 0, "att_minimise takes Euler poses (pose_format 0)");
  REQUIRE(steps >= 0, "steps = %d < 0", steps);
  REQUIRE(pose_out_dev != nullptr || n_tiles == 0, "pose_out is NULL");
  REQUIRE(energy_dev != nullptr || n_tiles == 0, "energy output is NULL");
  REQUIRE(work_counter_dev != nullptr, "work counter is NULL");
  REQUIRE(cfg->beta1 >= 0.f && cfg->beta1 < 1.f && cfg->beta2 >= 0.f && cfg->beta2 < 1.f,
          "beta1/beta2 must be in [0, 1)");
  REQUIRE(cfg->step0 >= 0, "step0 < 0");
  p.pose_out = pose_out_dev;
  p.adam = adam_state_dev;
  p.energy = energy_dev;
  p.status = status_dev;
  p.counter = work_counter_dev;
  p.stats = stats_dev;
  p.steps = steps;
  p.lr_rot = cfg->lr_rot;
  p.lr_trans = cfg->lr_trans;
  p.b1 = cfg->beta1;
  p.b2 = cfg->beta2;
  p.eps = cfg->eps;
  p.step0 = cfg->step0;
  if (n_tiles == 0) return ATT_OK;
  int blocks = 0;
  rc = persistent_blocks(MODE_MIN, S, K, threads, p.rec_slot, launch, n_tiles, &blocks);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(work_counter_dev, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "att_minimise counter reset");
  e = launch_score(p, MODE_MIN, S, K, blocks, threads, st);
  if (e != cudaSuccess) return cuda_fail(e, "att_minimise launch");
  return ATT_OK;
}

extern "C" int att_minimise_schema(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                                   const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles,
                                   int n_pose_rows, const float* pose_in_dev, float* pose_out_dev, const int* pose_lig_dev,
                                   const AttSchemaCfg* cfg, float* energy_dev, int* status_dev,
                                   int* work_counter_dev, const AttLaunchCfg* launch, void* stream) {
  REQUIRE(cfg != nullptr, "schema cfg is NULL");
  KParams p;
  int S = 8, K = 1, threads = 128;
  int rc = fill_common(&p, grids, n_grids, ligs, segs_dev, n_segs, seg_tile_dev, n_tiles, n_pose_rows, pose_in_dev,
                       pose_lig_dev, &cfg->eval, launch, &S, &K, &threads);
  if (rc) return rc;
  REQUIRE(cfg->n_stages >= 1 && cfg->n_stages <= ATT_MAX_STAGES, "n_stages = %d (1..%d)", cfg->n_stages,
          ATT_MAX_STAGES);
  int total = 0;
  for (int i = 0; i < cfg->n_stages; ++i) {
    REQUIRE(cfg->epochs[i] >= 0, "stage %d: epochs < 0", i);
    total += cfg->epochs[i];
  }
  REQUIRE(total >= 1, "the schema has no epochs");
  REQUIRE(cfg->beta1 >= 0.f && cfg->beta1 < 1.f && cfg->beta2 >= 0.f && cfg->beta2 < 1.f,
          "beta1/beta2 must be in [0, 1)");
  REQUIRE(pose_out_dev != nullptr || n_tiles == 0, "pose_out is NULL");
  REQUIRE(energy_dev != nullptr || n_tiles == 0, "energy output is NULL");
  REQUIRE(work_counter_dev != nullptr, "work counter is NULL");
  p.pose_out = pose_out_dev;
  p.energy = energy_dev;
  p.status = status_dev;
  p.counter = work_counter_dev;
  p.steps = total;
  p.b1 = cfg->beta1;
  p.b2 = cfg->beta2;
  p.eps = cfg->eps;
  p.eps_root = cfg->eps_root;
  p.qs_n = cfg->n_stages;
  for (int i = 0; i < ATT_MAX_STAGES; ++i) {
    p.qs_epochs[i] = i < cfg->n_stages ? cfg->epochs[i] : 0;
    p.qs_lr[i] = i < cfg->n_stages ? cfg->lr[i] : 0.f;
    p.qs_grav[i] = i < cfg->n_stages ? cfg->gravity[i] : 0;
  }
  if (n_tiles == 0) return ATT_OK;
  int blocks = 0;
  rc = persistent_blocks(MODE_QUAT, S, K, threads, p.rec_slot, launch, n_tiles, &blocks);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(work_counter_dev, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "att_minimise_schema counter reset");
  e = launch_score(p, MODE_QUAT, S, K, blocks, threads, st);
  if (e != cudaSuccess) return cuda_fail(e, "att_minimise_schema launch");
  return ATT_OK;
}

extern "C" int att_energrad_backward(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                                     const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles,
                                     int n_pose_rows, const float* pose_dev, const int* pose_lig_dev, const AttEvalCfg* cfg,
                                     const float* dL_dE_dev, float* dL_dpose_dev, float* dgrid_inner_dev,
                                     float* dgrid_outer_dev, const AttLaunchCfg* launch, void* stream) {
  KParams p;
  int S = 8, K = 1, threads = 128;
  int rc = fill_common(&p, grids, n_grids, ligs, segs_dev, n_segs, seg_tile_dev, n_tiles, n_pose_rows, pose_dev, pose_lig_dev,
                       cfg, launch, &S, &K, &threads);
  if (rc) return rc;
  REQUIRE(cfg->pose_format == 0, "att_energrad_backward takes Euler poses (pose_format 0)");
  REQUIRE(dL_dE_dev != nullptr || n_tiles == 0, "dL_dE is NULL");
  p.dLdE = dL_dE_dev;
  p.dLdpose = dL_dpose_dev;
  p.dgrid_inner = dgrid_inner_dev;
  p.dgrid_outer = dgrid_outer_dev;
  {
    const AttGridGeom& g = grids[0].geom;
    p.n_dgrid_inner = (long long)g.n_types * g.dim[0] * g.dim[1] * g.dim[2] * 4;
    p.n_dgrid_outer = (long long)g.n_types * g.dim2[0] * g.dim2[1] * g.dim2[2] * 4;
  }
  if (n_tiles == 0) return ATT_OK;
  const int wpb = threads / 32;
  const int blocks = (n_tiles + wpb - 1) / wpb;
  cudaError_t e = launch_score(p, MODE_BWD, S, K, blocks, threads, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_energrad_backward launch");
  return ATT_OK;
}

extern "C" int att_grid_repack(const AttGridGeom* geom, const float* inner_dev, const float* outer_dev,
                               void* bricks_dev, void* stream) {
  int rc = check_geom(geom);
  if (rc) return rc;
  REQUIRE(inner_dev != nullptr && bricks_dev != nullptr, "inner grid / bricks NULL");
  REQUIRE(aligned(inner_dev, 16) && aligned(bricks_dev, 128), "inner grid 16-B / bricks 128-B alignment");
  if (outer_dev != nullptr) {
    REQUIRE(aligned(outer_dev, 16), "outer grid not 16-B aligned");
    REQUIRE(geom->dim2[0] >= 2 && geom->dim2[1] >= 2 && geom->dim2[2] >= 2, "outer grid needs dim2 >= 2");
  }
  cudaError_t e = launch_repack(*geom, inner_dev, outer_dev, bricks_dev, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_grid_repack");
  return ATT_OK;
}

extern "C" int att_build_potential_grid(const AttGridGeom* geom, const float* rec_dev, int n_rec,
                                        const float* pair_dev, int n_rtypes, int n_ltypes, float cutoff, int outer,
                                        float* out_dev, void* stream) {
  int rc = check_geom(geom);
  if (rc) return rc;
  REQUIRE(n_rec >= 0 && (n_rec == 0 || rec_dev != nullptr), "receptor beads NULL");
  REQUIRE(pair_dev != nullptr && out_dev != nullptr, "pair table / output NULL");
  REQUIRE(n_rtypes >= 1 && n_ltypes >= 1 && n_ltypes <= 65535, "type counts out of range");
  REQUIRE(cutoff > 0.f, "cutoff must be > 0");
  REQUIRE(outer == 0 || (geom->dim2[0] >= 1 && geom->dim2[1] >= 1 && geom->dim2[2] >= 1), "outer grid needs dim2");
  REQUIRE(aligned(out_dev, 16) && aligned(pair_dev, 16) && (n_rec == 0 || aligned(rec_dev, 16)), "alignment");
  cudaError_t e = launch_build_potential(*geom, rec_dev, n_rec, pair_dev, n_rtypes, n_ltypes, cutoff, outer,
                                         out_dev, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_build_potential_grid");
  return ATT_OK;
}

extern "C" int att_nbgrid_pack_records(const uint32_t* hdr_dev, const uint16_t* list_dev, long long n_voxels,
                                       int rec_bytes, void* records_dev, void* stream) {
  REQUIRE(rec_bytes == 32 || rec_bytes == 64 || rec_bytes == 128, "rec_bytes = %d (32, 64 or 128)", rec_bytes);
  REQUIRE(n_voxels >= 0, "n_voxels < 0");
  REQUIRE(hdr_dev != nullptr && list_dev != nullptr && records_dev != nullptr, "hdr / list / records NULL");
  REQUIRE(aligned(hdr_dev, 8) && aligned(records_dev, 16), "hdr 8-B / records 16-B alignment");
  if (n_voxels == 0) return ATT_OK;
  cudaError_t e = launch_nb_pack(hdr_dev, list_dev, n_voxels, rec_bytes, records_dev, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_nbgrid_pack_records");
  return ATT_OK;
}

extern "C" int att_kernel_debug_info(unsigned long long* info3, int clear, void* stream) {
  REQUIRE(info3 != nullptr, "info3 is NULL");
  cudaError_t e = kernel_debug_info(info3, clear, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_kernel_debug_info");
  return ATT_OK;
}

extern "C" int att_kernel_status(int* error_word, int clear, void* stream) {
  REQUIRE(error_word != nullptr, "error_word is NULL");
  cudaError_t e = kernel_status(error_word, clear, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_kernel_status");
  return ATT_OK;
}

extern "C" long long att_nbgrid_workspace_bytes(long long n_voxels) { return nb_workspace_bytes(n_voxels); }

extern "C" int att_nbgrid_count(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                                uint32_t* hdr_dev, unsigned long long* total_dev, void* workspace_dev,
                                long long workspace_bytes, void* stream) {
  int rc = check_geom(geom);
  if (rc) return rc;
  const long long nvox = (long long)geom->dim[0] * geom->dim[1] * geom->dim[2];
  REQUIRE(n_rec >= 0 && n_rec < (int)ATT_NB_EMPTY && (n_rec == 0 || rec_dev != nullptr), "receptor beads");
  REQUIRE(hdr_dev != nullptr && total_dev != nullptr && workspace_dev != nullptr, "NULL output / workspace");
  REQUIRE(workspace_bytes >= nb_workspace_bytes(nvox), "workspace of %lld bytes < %lld", workspace_bytes,
          nb_workspace_bytes(nvox));
  REQUIRE(radius >= 0.f, "radius < 0");
  cudaError_t e = launch_nb_count(*geom, rec_dev, n_rec, radius, hdr_dev, total_dev, workspace_dev,
                                  (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_nbgrid_count");
  return ATT_OK;
}

extern "C" int att_nbgrid_fill(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                               const uint32_t* hdr_dev, uint16_t* list_dev, void* stream) {
  int rc = check_geom(geom);
  if (rc) return rc;
  REQUIRE(n_rec >= 0 && n_rec < (int)ATT_NB_EMPTY && (n_rec == 0 || rec_dev != nullptr), "receptor beads");
  REQUIRE(hdr_dev != nullptr && list_dev != nullptr, "hdr / list NULL");
  cudaError_t e = launch_nb_fill(*geom, rec_dev, n_rec, radius, hdr_dev, list_dev, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "att_nbgrid_fill");
  return ATT_OK;
}
