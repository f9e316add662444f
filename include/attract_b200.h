/*
 * attract_b200 -- C ABI of the B200 (sm_100a) ATTRACT scoring + rigid-body
 * minimisation path.
 *
 * Every pointer named *_dev is a caller-owned device buffer; the library does
 * not allocate device memory.  Every call is asynchronous on the given CUDA
 * stream and returns an int status: ATT_OK (0) or an ATT_E_* code, with a
 * message in att_last_error_string() (thread-local).  Nothing aborts or traps.
 *
 * Reference interface each entry point replaces (paths within
 * sjdv1982/attract-jax):
 *   att_energrad         main()/main0() + value_and_grad,  test5.py:404-429
 *                        (and the 4x4-matrix form of test1.py:361-366,409-412)
 *   att_minimise         the batch/epoch optimiser loop, test5.py:436-467
 *                        (optax.adam form of test4.py:440-455)
 *   att_minimise_schema  the same loop with test5's own protocol: quaternion
 *                        poses, optax.adabelief, the SCHEMA stages, test5.py:14-23,445-467
 *   att_energrad_backward  reverse mode of test5.py:429, extended to the grid
 *                        values (no counterpart: JAX never differentiates the grid)
 *   att_grid_repack      the dense grid arrays of read_grid2.py:92-155
 *                        -> the brick layout the kernels read
 *   att_build_potential_grid  calc_grid(), test-calc-grid-energy.py:154-196
 *   att_nbgrid_count / att_nbgrid_fill  the neighbour lists of
 *                        test-calc-grid-energy.py:90-103 (KD-tree query)
 */
#ifndef ATTRACT_B200_H
#define ATTRACT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATT_OK 0
#define ATT_E_INVALID 1     /* bad argument (shape, range, alignment, NULL) */
#define ATT_E_CUDA 2        /* a CUDA runtime call failed */
#define ATT_E_UNSUPPORTED 3 /* configuration not built into this library */

#define ATT_MAX_GRIDS 8
#define ATT_NB_EMPTY 65535u /* empty neighbour-list slot (read_grid2.py:118) */

/* grad_mode */
#define ATT_GRAD_REFERENCE 0 /* grid gradient = -interpolated stored force (test5.py:310),
                                nb gradient with the plateau correction (test5.py:220-229) */
#define ATT_GRAD_ANALYTIC 1  /* exact derivative of the computed energy */

/* flags */
#define ATT_FLAG_TRILINEAR_QUIRK 1 /* reference floor/ceil weights: a bead with an exactly
                                      integer voxel coordinate reads 0 (test5.py:256-259) */

/* per-pose status bits written by att_minimise / att_energrad */
#define ATT_STATUS_NONFINITE_GRAD 1   /* a step saw a non-finite gradient and was skipped */
#define ATT_STATUS_NONFINITE_ENERGY 2 /* the returned energy is not finite */
#define ATT_STATUS_NONFINITE_POSE 4   /* the input pose has a non-finite component */

/* device-wide kernel error word (att_kernel_status) */
#define ATT_KERR_COPY_TIMEOUT 1 /* reserved: no kernel of this build waits on a flag or another thread (a
                                   lane waits only for its own cp.async copies and at warp barriers), so
                                   none can time out */
#define ATT_KERR_BOUNDS 2       /* (ATT_BOUNDS_CHECK builds) an index failed its check; the access was skipped */
#define ATT_KERR_BAD_SEGMENT 4  /* a segment named a missing grid or ligand or reached beyond n_pose_rows, or a
                                   pose's conformer index (pose_lig) or its ligand's bead range left the ligand
                                   set: those poses were skipped (outputs unwritten), checked before any access */

/* A pose is served by lanes_per_pose lanes holding up to 8 beads each; a
   ligand with more than 8 * lanes_per_pose beads is evaluated in chunks of that
   many beads (slower: its coordinates are re-read every chunk). */
#define ATT_MAX_BEADS_PER_LANE 8

/* Geometry of one receptor grid: the scalar fields of read_grid2.py's Grid. */
typedef struct AttGridGeom {
  float origin[3];  /* position of inner grid point (0,0,0) */
  float spacing;    /* gridspacing (inner); the outer grid has 2*spacing */
  int dim[3];       /* inner grid points per axis */
  int dim2[3];      /* outer grid points per axis */
  int extension;    /* gridextension: outer point j sits at origin + (2j - extension)*spacing */
  float plateau;    /* plateaudis: pair terms apply for d < plateau */
  int n_types;      /* potential slots (ligand grid types) */
  int pad_;
} AttGridGeom;

/* One receptor, resident on the device (all pointers *_dev). */
typedef struct AttGrid {
  AttGridGeom geom;
  const void* bricks;          /* float4 [n_types][n_inner_bricks + n_outer_bricks][8]; 128-B aligned;
                                  NULL = no potential grid (neighbour grid only) */
  long long n_inner_bricks;    /* (dim[0]-1)(dim[1]-1)(dim[2]-1) */
  long long n_outer_bricks;    /* (dim2[0]-1)(dim2[1]-1)(dim2[2]-1), 0 = no outer grid */
  const uint32_t* nb_hdr;      /* [list-grid points][2] = {start, count} per point (CSR; the list grid
                                  is the inner grid unless nb_refine > 1); NULL = no neighbour grid */
  const uint16_t* nb_list;     /* receptor bead index per entry (ATT_NB_EMPTY skipped) */
  long long n_nb_entries;
  const float* rec;            /* [n_rec][4] x, y, z, receptor type (as an int32 bit pattern) */
  int n_rec;
  int n_rtypes;                /* receptor types in the pair table */
  int n_ltypes;                /* ligand types in the pair table */
  int nb_rec_bytes;            /* 32, 64 or 128: size of one neighbour record (below) */
  const float* pair;           /* [n_ltypes][n_rtypes][8], 32-B aligned: rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2 */
  const void* nb_rec;          /* one neighbour record per list-grid point, 16-B aligned
                                  (att_nbgrid_pack_records): the first (nb_rec_bytes - 6) / 2
                                  entries inline (u16 each, from byte 0), the u16 count at byte
                                  nb_rec_bytes - 6, the u32 overflow index into nb_list at byte
                                  nb_rec_bytes - 4; required with nb_hdr */
  int nb_refine;               /* 0 or 1: the lists sit at the inner grid points (the reference's
                                  neighbour grid); 2 or 4: at the points of the inner grid refined
                                  that many times per axis (spacing / r, (dim - 1) * r + 1 points per
                                  axis, same origin), which nb_hdr and nb_rec then index.  A bead
                                  inside the inner grid reads the list of its nearest list-grid
                                  point; lists that hold every receptor bead within plateau + the
                                  list spacing * sqrt(3) / 2 give the same pairs at every r, with
                                  fewer entries beyond the plateau for larger r. */
  int pad2_;
} AttGrid;

/* Inline entries of a neighbour record of `bytes` bytes. */
#define ATT_NB_INLINE(bytes) (((bytes) - 6) / 2)

/* Ligands: all beads of all ligands concatenated. */
typedef struct AttLigands {
  const float* beads;   /* [n_beads][4] x, y, z, type word = gtype | (ltype << 16) (int32 bits) */
  const int* offset;    /* [n_lig + 1] first bead of each ligand */
  int n_lig;
  int max_beads;        /* max over ligands of offset[l+1]-offset[l] */
  int n_beads;          /* rows of beads; a ligand whose offsets leave [0, n_beads] is skipped */
  int pad_;
} AttLigands;

/* A run of consecutive poses scored against one grid with one ligand. */
typedef struct AttSegment {
  int grid;     /* index into the grids array */
  int lig;      /* ligand index (base index when pose_lig is given) */
  int pose0;    /* first pose of the run */
  int n_poses;
  int step0;    /* ADAM steps these poses' adam_state has already taken (added to
                   AttAdamCfg.step0): runs at different stages share one launch */
  int pad_[3];
} AttSegment;

typedef struct AttEvalCfg {
  int grad_mode;    /* ATT_GRAD_* */
  int flags;        /* ATT_FLAG_* */
  float gravity;    /* adds gravity*|t|^2 (test5.py:419 uses 0.1) */
  int pose_format;  /* 0: [B][6] phi,psi,theta,tx,ty,tz ; 1: [B][16] row-vector 4x4 (test5.py:413-415) */
} AttEvalCfg;

typedef struct AttAdamCfg {
  AttEvalCfg eval;
  float lr_rot;     /* rad */
  float lr_trans;   /* Angstrom */
  float beta1, beta2, eps;
  int step0;        /* steps already taken by the given adam_state (bias correction) */
} AttAdamCfg;

/* The minimisation protocol of test5.py:14-23,436-467: stages of (epochs,
   learning rate, gravity on/off), each with a fresh optax.adabelief state over
   the (quaternion, translation) pose. */
#define ATT_MAX_STAGES 8
typedef struct AttSchemaCfg {
  AttEvalCfg eval;          /* grad_mode, flags; gravity = weight of |t|^2 in stages with gravity on
                               (test5.py:419: 0.1); pose_format ignored */
  int n_stages;             /* 1..ATT_MAX_STAGES */
  int epochs[ATT_MAX_STAGES];
  float lr[ATT_MAX_STAGES];
  int gravity[ATT_MAX_STAGES];
  float beta1, beta2, eps, eps_root;  /* optax.adabelief defaults: 0.9, 0.999, 1e-16, 1e-16 */
} AttSchemaCfg;

/* Launch shape; zeros pick the defaults / autotuned values. */
typedef struct AttLaunchCfg {
  int lanes_per_pose;   /* 8, 16 or 32 (poses per warp = 32 / lanes_per_pose) */
  int block_threads;    /* 32, 64, 96 or 128 (0 = the largest whose shared memory fits) */
  int blocks;           /* persistent CTAs (att_minimise), 0 = fill the GPU */
  int test_flags;       /* reserved: must be 0 */
} AttLaunchCfg;


const char* att_last_error_string(void);
const char* att_version(void);

/* Bytes of float4 bricks needed for a grid: n_types*(n_inner+n_outer)*128. */
long long att_grid_brick_bytes(const AttGridGeom* geom, int with_outer);

/* Dense reference grids -> bricks.  inner_dev: float [n_types][dim0][dim1][dim2][4],
   outer_dev: [n_types][dim2_0][dim2_1][dim2_2][4] or NULL.  (read_grid2.py:92-155) */
int att_grid_repack(const AttGridGeom* geom, const float* inner_dev, const float* outer_dev,
                    void* bricks_dev, void* stream);

/* Arguments shared by the scoring entry points below: segs_dev [n_segs] and
   seg_tile_dev [n_segs+1] (first work tile of each segment; a tile is
   32/lanes_per_pose consecutive poses of one segment) on the device;
   n_pose_rows = B, the rows of the pose and per-pose output arrays.  The
   kernels check every segment (grid < n_grids, lig < ligs->n_lig, pose0 >= 0,
   pose0 + n_poses <= B), every conformer index (pose_lig) and every ligand's
   bead range (within ligs->n_beads, at most ligs->max_beads beads) before any
   access; a pose that fails is skipped, its outputs stay unwritten, and
   ATT_KERR_BAD_SEGMENT is set in the device error word (att_kernel_status).

   One energy (+gradient) evaluation of every pose of every segment.
   pose_dev [B][6] (or [B][16]); pose_lig_dev [B] optional per-pose ligand offset (conformers);
   energy_dev [B]; grad_dev [B][6] (Euler) or [B][16] dE/dmat (pose_format 1), may be NULL;
   status_dev [B] optional.  test5.py:404-429. */
int att_energrad(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                 const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows,
                 const float* pose_dev, const int* pose_lig_dev, const AttEvalCfg* cfg,
                 float* energy_dev, float* grad_dev, int* status_dev,
                 const AttLaunchCfg* launch, void* stream);

/* Fused rigid-body ADAM minimisation: `steps` evaluate+update iterations, then a
   final evaluation whose energy is returned.  pose_in_dev/pose_out_dev [B][6] (may
   alias); adam_state_dev [B][12] (m[6], v[6]) in/out or NULL (start from zero);
   work_counter_dev: one int of scratch, zeroed by this call; stats_dev: optional
   [5] u64 counters, added to (bead evaluations with a grid brick, neighbour
   lookups, list entries visited, brick copies, record copies; a bead copies its
   brick or record only when it differs from the one its slot holds).
   seg_tile_dev [n_segs+1]: first work tile of each segment (a tile is
   32/lanes_per_pose consecutive poses of one segment).  test5.py:436-467. */
int att_minimise(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                 const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows,
                 const float* pose_in_dev, float* pose_out_dev, const int* pose_lig_dev,
                 float* adam_state_dev, const AttAdamCfg* cfg, int steps,
                 float* energy_dev, int* status_dev, int* work_counter_dev,
                 unsigned long long* stats_dev, const AttLaunchCfg* launch, void* stream);

/* The whole SCHEMA protocol (test5.py:445-467) as one persistent launch:
   pose_in_dev / pose_out_dev [B][8] = qx, qy, qz, qw (scalar last), tx, ty,
   tz, unused (may alias).  The input quaternion is normalised
   (Rotation.from_quat); every epoch evaluates E and dE/d(q, t) -- dE/dq through
   Rotation.as_matrix's homogeneous quaternion form -- applies the adabelief
   update (prediction error against the previous first moment, as optax's
   scale_by_belief) and renormalises the quaternion.  energy_dev [B] receives
   the energy of the last evaluation, before the last update, as the reference
   reports it (test5.py:465).  A step with a non-finite gradient is skipped and
   flagged in status_dev.  work_counter_dev: one int of scratch. */
int att_minimise_schema(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                        const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows,
                        const float* pose_in_dev, float* pose_out_dev, const int* pose_lig_dev,
                        const AttSchemaCfg* cfg, float* energy_dev, int* status_dev, int* work_counter_dev,
                        const AttLaunchCfg* launch, void* stream);

/* Adjoint of att_energrad for L = sum_b dL_dE[b] * E[b]: dL/dpose [B][6] and the
   scatter-add of dL/d(grid energy values) into dgrid_inner_dev / dgrid_outer_dev,
   float [n_types][dim..][4] (channel 0 receives the gradient; the caller zeroes
   the buffers).  Recomputes the forward instead of storing per-bead weights. */
int att_energrad_backward(const AttGrid* grids, int n_grids, const AttLigands* ligs,
                          const AttSegment* segs_dev, int n_segs, const int* seg_tile_dev, int n_tiles, int n_pose_rows,
                          const float* pose_dev, const int* pose_lig_dev, const AttEvalCfg* cfg,
                          const float* dL_dE_dev, float* dL_dpose_dev,
                          float* dgrid_inner_dev, float* dgrid_outer_dev,
                          const AttLaunchCfg* launch, void* stream);

/* Potential grid of energies and forces for ligand types 0..n_ltypes-1 at the inner
   (outer=0) or outer (outer=1) grid points: per receptor bead within `cutoff`,
   the pair energy and force beyond the plateau, the plateau energy and the plateau
   force along d inside it.  pair_dev as in AttGrid.pair but carrying the plateau
   values of this geometry.  out_dev float [n_ltypes][dim..][4].
   test-calc-grid-energy.py:154-196. */
int att_build_potential_grid(const AttGridGeom* geom, const float* rec_dev, int n_rec,
                             const float* pair_dev, int n_rtypes, int n_ltypes, float cutoff,
                             int outer, float* out_dev, void* stream);

/* Neighbour lists of receptor beads within `radius` of every inner grid point,
   ascending bead index.  att_nbgrid_count writes hdr_dev [V][2] = {start, count}
   and the entry total (one u64 on the device); it needs
   att_nbgrid_workspace_bytes(V) bytes of scratch.  att_nbgrid_fill then writes
   the entries.  The starts are 32-bit: a total above 2^32 - 1 (the u64 at
   total_dev holds the true count) means they wrapped, and the caller must not
   fill or use the lists.  A point is within the radius when
   fl(fl(fl(dx*dx) + fl(dy*dy)) + fl(dz*dz)) <= fl(radius*radius), each float32
   operation rounded on its own (dx = fl(x - rx), x = fl(origin + fl(i*spacing))),
   so a host restatement reproduces the lists bit for bit.
   test-calc-grid-energy.py:90-103. */
long long att_nbgrid_workspace_bytes(long long n_voxels);
int att_nbgrid_count(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                     uint32_t* hdr_dev, unsigned long long* total_dev, void* workspace_dev,
                     long long workspace_bytes, void* stream);
int att_nbgrid_fill(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                    const uint32_t* hdr_dev, uint16_t* list_dev, void* stream);

/* Fixed-size neighbour records from the CSR lists: record v holds
   {first `inline` entries (rest ATT_NB_EMPTY), count, overflow index = start
   + inline} in the layout of AttGrid.nb_rec (entries first, so that the
   kernels read eight per 16-byte load); entries beyond the inline ones stay
   in the CSR list, which the kernels keep reading.  A record is copied into
   shared memory (16-byte cp.async pieces) when a bead's nearest list-grid
   point changes.
   records_dev: n_voxels * rec_bytes bytes, 16-B aligned; rec_bytes 32/64/128.
   (No counterpart in the reference: a layout of the neighbour grid of
   read_grid2.py:113-124 for the B200 kernels.) */
int att_nbgrid_pack_records(const uint32_t* hdr_dev, const uint16_t* list_dev, long long n_voxels,
                            int rec_bytes, void* records_dev, void* stream);

/* att_nbgrid_count without a caller workspace.  No counterpart in the
   reference (its neighbour lists come from a KD-tree on the host).
   Some callers of this library cannot allocate device memory: a plugin that
   only receives the buffers of a host framework owning all GPU memory through
   its own allocator, a C/FFI binding with no allocator of its own, or a
   latency-bound service that must never call cudaMalloc/cudaFree (they
   synchronise the device).  This entry point takes the same inputs and
   outputs as att_nbgrid_count but keeps the scan workspace in a fixed array
   inside the library (32 KB on every device that loads it, held until exit),
   so it allocates nothing: grids of at most ATT_NBGRID_NOALLOC_MAX_VOXELS inner
   points; larger grids are rejected with ATT_E_INVALID.  The first call on a
   device looks up the array's device address (cudaGetSymbolAddress) with that
   device current; make that first call before any stream capture.  All calls
   share the one array: calls that overlap on the GPU (other streams, other
   host threads) race on it and must be serialised by the caller. */
#define ATT_NBGRID_NOALLOC_MAX_VOXELS (8192LL * 1024LL)
int att_nbgrid_count_noalloc(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                             uint32_t* hdr_dev, unsigned long long* total_dev, void* stream);

/* Explicit all-pairs ATTRACT energy without grids: for every pose, the sum
   over every (ligand bead, receptor bead) pair with d < rcut (rcut = 0: all
   pairs) of the pair potential of `pair_dev` (same layout as AttGrid.pair;
   give it eplat = 0 for the plain potential).  rec_dev [n_rec][4] x, y, z,
   receptor type (int32 bits); lig_dev [n_lig][4] x, y, z, ligand type (int32
   bits); pose_dev [B][6] (pose_format 0) or [B][16] row-vector 4x4 (1);
   energy_dev [B]; grad_dev [B][6] dE/d(Euler, t) or [B][16] dE/dmat, may be
   NULL.  Receptor beads grouped by type run faster (a pair-parameter row is
   reloaded only where the receptor type changes); the result does not depend
   on their order beyond float32 summation order.  Replaces main() of
   test-energy.py:46-58 (the reference's rescoring; ATTRACT --score with --rcut). */
int att_allpairs_energy(const float* rec_dev, int n_rec, const float* lig_dev, int n_lig,
                        const float* pose_dev, int n_poses, int pose_format, const float* pair_dev,
                        int n_rtypes, int n_ltypes, float rcut, float* energy_dev, float* grad_dev,
                        void* stream);

/* Read the device-wide error word of the scoring kernels (ATT_KERR_* bits, 0 =
   none) into *error_word, clearing it if `clear`; synchronises `stream`.  A
   non-zero word means some warp stopped early and its poses' outputs are stale.
   (No counterpart in the reference: JAX has no device-side waits.) */
int att_kernel_status(int* error_word, int clear, void* stream);

/* Debug builds (-DATT_BOUNDS_CHECK): the first failed index check of the
   scoring kernels as {check code, index, bound} (zeros if none, and always in
   regular builds); cleared if `clear`; synchronises `stream`. */
int att_kernel_debug_info(unsigned long long* info3, int clear, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ATTRACT_B200_H */
