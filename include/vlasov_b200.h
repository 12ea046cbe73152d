/*
 * vlasov_b200.h -- C ABI of the B200 (sm_100a) library that serves the
 * per-step pseudo-particle loop of LaurentPlagne/Vlasov.jl.
 *
 * The entry points are the calls the reference's host makes on its device
 * accelerator (src/accelerator.jl, src/devicemesh.jl, src/simulation.jl),
 * flattened to plain pointers and sizes.  Each declaration names the
 * reference interface it replaces.
 *
 * Conventions
 *   - Every function returns an int: 0 on success, a negative VLB_ERR_* code
 *     otherwise; vlb_last_error() gives a message (thread-local).  Nothing
 *     throws or aborts across this boundary.
 *   - The library owns every device allocation (the opaque vlb_ctx); the
 *     caller owns every host pointer it passes, and each call copies.
 *   - All work of a context runs on one library-owned CUDA stream.  Calls that
 *     return host values synchronise that stream; the others are ordered on
 *     it.  A context is not re-entrant; separate contexts are independent.
 *   - Particles are held as the reference's packed form (PackedParticle,
 *     src/particles.jl:86-91): per axis the 1-based nearest fine knot `k`
 *     (int32, unclamped) and the offset `delta` from it (float32), for the
 *     current and the previous position.  Host arrays are structure-of-arrays
 *     of length 3*npart: all x, then all y, then all z.
 *   - Cells are 0-based: cell = (kx-1) + nk*((ky-1) + nk*(kz-1)) with each k
 *     clamped to [1, nk] (src/kernels.jl:902-908 minus one).
 *   - Grids are n^3 float32 arrays, i fastest (the reference's column-major
 *     (i,j,k) layout).
 */
#ifndef VLASOV_B200_H
#define VLASOV_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define VLB_API __attribute__((visibility("default")))
#else
#define VLB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define VLB_OK 0
#define VLB_ERR_ARG (-1)      /* bad size, null handle, non-uniform axis ... */
#define VLB_ERR_CUDA (-2)     /* a CUDA call failed */
#define VLB_ERR_STATE (-3)    /* call out of order (e.g. forces before a sort) */
#define VLB_ERR_TIMEOUT (-4)  /* a bounded device wait gave up */
#define VLB_ERR_NOMEM (-5)

typedef struct vlb_ctx vlb_ctx;

/* One cubic mesh level: the tables of SplineMesh (src/mesh.jl:327-382) that
 * the step reads, in float64 (converted to float32 on upload, as DeviceMesh
 * does, src/devicemesh.jl:49-81).  The three axes of a level are identical. */
typedef struct vlb_level_desc {
  int32_t nknots;              /* knots per axis; n = 2*nknots points per axis */
  const double* knots;         /* [nknots] */
  const double* colloc;        /* [n] collocation points */
  const double* sinv;          /* [n*n] row-major S^-1 (src/collocation.jl:53) */
  const double* laplacian;     /* [n*n] row-major D = S'' S^-1 (src/collocation.jl:94) */
  const double* eigvec;        /* [(n-2)^2] row-major M of D[2:end-1,2:end-1] */
  const double* eigvec_inv;    /* [(n-2)^2] row-major M^-1 */
  const double* eigval;        /* [n-2] real eigenvalues */
  const double* dual_moments;  /* [3*n] S^-T m_k, k = 0,1,2 (src/mesh.jl:367-368) */
  const double* dual_lengths;  /* [n] (src/deposition.jl:23-33) */
  double locate_x0;            /* LocateTable (src/splines.jl:362-376) */
  double locate_invwidth;
  int32_t locate_ncells;
  const int32_t* locate_cells; /* [locate_ncells], 1-based cells */
} vlb_level_desc;

/* GaussianSmoothing tables (src/fields.jl:44-53), column-major: the values of
 * one table column are contiguous. */
typedef struct vlb_smoothing_desc {
  int32_t nbdt;                /* columns - 1 (1000) */
  double spacing;              /* fine step h */
  const double* overlap;       /* [(nbdt+1)*10] */
  const double* gradient;      /* [(nbdt+1)*10] */
  const double* nodes;         /* [(nbdt+1)*8] */
} vlb_smoothing_desc;

typedef struct vlb_config {
  int64_t npart;
  double weight;               /* electrons carried by one pseudo-particle */
  vlb_level_desc fine;         /* uniform axis */
  vlb_level_desc coarse;       /* stretched axis */
  vlb_smoothing_desc smoothing;
  int32_t device;              /* CUDA device ordinal */
  int32_t flags;               /* reserved, 0 */
} vlb_config;

/* How the projectile's Coulomb force is softened (vlb_projectile.softening).
 * The reference's two paths differ here:
 *   VLB_SOFTENING_DEVICE: its resident device path.  Particles whose 10^3
 *     stencil fits take a Gaussian of width `sigma` (gaussian_force_kernel,
 *     src/accelerator.jl:632, src/kernels.jl:425-443) at the position rebuilt
 *     from their cell's clamped knots, and the projectile sums that Gaussian
 *     reaction over every particle; out-of-stencil particles take the ball of
 *     radius `ball_radius` on their own force (src/accelerator.jl:719-723).
 *     e_electrons = w q sum erf(r / sqrt(2) sigma) / r.
 *   VLB_SOFTENING_BALL: its CPU path, projectile_forces! with BallSoftening
 *     (src/projectile.jl:79-80, 203-232): the uniform ball of radius
 *     `ball_radius` for every particle, both ways, at the particle's own
 *     position.  e_electrons = w sum uniform_sphere_potential(q, R, r)
 *     (src/meanfield.jl:52-54). */
#define VLB_SOFTENING_DEVICE 0
#define VLB_SOFTENING_BALL 1

/* Projectile state (src/projectile.jl:141-150).  `sigma` is the width of
 * the Gaussian kernel the fused force path uses, scale(softening)
 * (src/accelerator.jl:632); `ball_radius` the radius of the ball softening
 * (the out-of-stencil particles' in VLB_SOFTENING_DEVICE, everyone's in
 * VLB_SOFTENING_BALL). */
typedef struct vlb_projectile {
  double position[3];
  double previous[3];
  double velocity[3];
  double charge;
  double mass;
  double sigma;
  double ball_radius;
  int32_t active;              /* 0: isolated cluster, no projectile */
  int32_t softening;           /* VLB_SOFTENING_DEVICE (0) or VLB_SOFTENING_BALL */
} vlb_projectile;

/* Parameters of one fused step (step!(sim; energy=false), src/simulation.jl:382-416). */
typedef struct vlb_step_params {
  double dt;
  double rcmax;                /* radius beyond which a particle counts as gone */
  double jellium_nions;        /* Jellium (src/meanfield.jl:332-340) */
  double jellium_radius;
  double capture_radius;       /* q(<R) around the projectile after the step; <= 0 skips */
  int32_t deposit_mode;        /* VLB_DEPOSIT_FLOAT32 or VLB_DEPOSIT_FIXED64 */
  int32_t advance_projectile;  /* 0 during priming (src/simulation.jl:254) */
  int32_t push;                /* 0: forces only, no Verlet (priming) */
  int32_t use_graph;           /* 1: replay the step as one captured CUDA graph */
  int32_t poisson_precision;   /* VLB_POISSON_FP32, _3XTF32 or _BF16X3, every mode product of the step */
  int32_t denoise;             /* 1: the learned denoiser on the fine density (vlb_set_denoiser) */
  int32_t energy;              /* 1: the energy budget's two sums (step!(sim; energy=true)) */
  int32_t film;                /* 1: append a film frame after the step (vlb_film_reserve) */
} vlb_step_params;

/* Device-side error flags (vlb_step_result.status, vlb_dn_status). */
#define VLB_STATUS_SCAN_TIMEOUT 1  /* a look-back scan gave up waiting */
#define VLB_STATUS_BAD_CELL 2      /* a particle outside the coarse deposit's cell table */
#define VLB_STATUS_OVERFLOW 4      /* a fixed-point accumulator out of range */
#define VLB_STATUS_MMA_TIMEOUT 8   /* a tensor-core kernel gave up waiting on its copies or MMAs */

#define VLB_DEPOSIT_FLOAT32 0
#define VLB_DEPOSIT_FIXED64 1   /* int64 fixed point, charge scaled by 2^40 */

typedef struct vlb_step_result {
  double kinetic;              /* step!(cloud, dt, acc) diagnostics */
  double escaped;
  double angular[3];
  double projectile_force[3];  /* projectile_forces!(..., acc) */
  double e_electrons;
  double e_jellium;
  double enclosed_charge;      /* q(<capture_radius) after the step */
  double total_charge;         /* fine charge before renormalisation */
  int32_t nout;                /* outside the fine deposit window */
  int32_t outcount;            /* 10^3 stencil leaves the fine grid */
  int32_t noccupied;           /* occupied fine cells */
  int32_t status;              /* device-side error flags (VLB_STATUS_*), 0 when clean */
  int32_t denoised;            /* 1: the step used the denoiser's density, 0: the deposit's */
  int32_t sort_path;           /* the step's sort: 1 the single-pass placement of a cloud still in
                                  its last sort's order (every particle within one cell of its old
                                  one), 2 that placement given up for the radix passes (a particle
                                  moved further), 0 the radix passes alone (no earlier order) */
  double hartree;              /* energy steps: 1/2 sum w phi_H at the step's positions (src/simulation.jl:511) */
  double interaction;          /* energy steps: sum w phi at the advanced positions (src/simulation.jl:393) */
} vlb_step_result;

/* Grid selectors for vlb_get_grid / vlb_set_grid. */
#define VLB_GRID_RHO_FINE 0
#define VLB_GRID_RHO_COARSE 1
#define VLB_GRID_PHI_FINE 2
#define VLB_GRID_PHI_COARSE 3
#define VLB_GRID_CSOL_FINE 4
#define VLB_GRID_CSOL_COARSE 5
#define VLB_GRID_CSOL_HARTREE_FINE 6    /* S^-1 phi_H of the last step run with params.energy */
#define VLB_GRID_CSOL_HARTREE_COARSE 7  /* S^-1 phi_H of the last solve */

/* Precision of the mode products (the tensor solves and the S^-1 conversions):
 * FP32 on the CUDA cores, or split-precision 3xTF32 on the tensor cores with
 * FP32 accumulation (even n <= 144 points per axis). */
#define VLB_POISSON_FP32 0
#define VLB_POISSON_3XTF32 1
#define VLB_POISSON_BF16X3 2

VLB_API const char* vlb_last_error(void);
VLB_API const char* vlb_version(void);

/* DeviceState(backend, E, meshes, sm, npart; packed=true)
 * (src/simulation.jl:104-115) + DeviceAccelerator (src/accelerator.jl:281-331):
 * uploads every table once and allocates the run's buffers. */
VLB_API int vlb_create(const vlb_config* cfg, vlb_ctx** out);
VLB_API int vlb_destroy(vlb_ctx* ctx);

/* upload!(acc.particles) / download!(acc.particles, backend)
 * (src/accelerator.jl:48-68).  SoA host arrays of 3*npart. */
VLB_API int vlb_upload_particles(vlb_ctx* ctx, const int32_t* knode, const float* delta,
                         const int32_t* pknode, const float* pdelta);
VLB_API int vlb_download_particles(vlb_ctx* ctx, int32_t* knode, float* delta,
                           int32_t* pknode, float* pdelta);

/* The same for the slots [first, first + count) of the cloud, host SoA arrays
 * of 3*count: the chunked transfers of a cloud built or read a slice at a
 * time (the construction of src/simulation.jl:171-216 and its priming,
 * src/simulation.jl:233-277, without a whole host copy of the cloud).
 * Slots out of [0, npart) return VLB_ERR_ARG. */
VLB_API int vlb_upload_particles_range(vlb_ctx* ctx, int64_t first, int64_t count, const int32_t* knode,
                               const float* delta, const int32_t* pknode, const float* pdelta);
VLB_API int vlb_download_particles_range(vlb_ctx* ctx, int64_t first, int64_t count, int32_t* knode,
                                 float* delta, int32_t* pknode, float* pdelta);

/* _pack!(acc, ::PackedPositions) -> _sort_and_list! (src/accelerator.jl:360-387,
 * 466-503): stable counting sort of the cloud by cell (the particles are
 * moved), occupied-cell list, bounds, out-of-stencil list.  Returns the
 * number of occupied cells and the out-of-stencil count. */
VLB_API int vlb_sort(vlb_ctx* ctx, int32_t* noccupied, int32_t* outcount);

/* The sort's products, for inspection: perm[s] = index before the sort of
 * the particle now in slot s; occupied[g] (0-based cells, increasing);
 * bounds[g] .. bounds[g+1] the slots of occupied cell g (bounds[0] = 0);
 * outlist[t] increasing slots whose stencil leaves the fine grid.  Any
 * pointer may be NULL.  Sizes: npart, noccupied, noccupied+1, outcount. */
VLB_API int vlb_get_sort(vlb_ctx* ctx, int32_t* perm, int32_t* occupied, int32_t* bounds,
                 int32_t* outlist);

/* The sizes vlb_get_sort writes for the last sort of the current cloud:
 * noccupied (occupied; bounds holds noccupied + 1) and outcount (outlist).
 * A caller that sorted through a step phase (vlb_step_deposit returns no
 * counts) reads them here before allocating.  Either pointer may be NULL. */
VLB_API int vlb_get_sort_sizes(vlb_ctx* ctx, int32_t* noccupied, int32_t* outcount);

/* deposit_smoothed!(rho, acc, mesh, sm, positions; charge)
 * (src/accelerator.jl:531-565): table columns, sorted 8^3 deposit, charge
 * renormalisation.  Needs vlb_sort.  `mode` is VLB_DEPOSIT_*.  Returns nout
 * and the charge before renormalisation. */
VLB_API int vlb_deposit_fine(vlb_ctx* ctx, double charge, int32_t mode, int32_t* nout,
                     double* total_charge);

/* deposit_cic!(rho, dm, acc, npart, charge, x0f, hf) (src/devicemesh.jl:93-106) */
VLB_API int vlb_deposit_coarse(vlb_ctx* ctx, double charge);

/* poisson!(phis, rhos, dms) (src/devicemesh.jl:160-169): coarse multipole
 * faces + solve, fine faces from the coarse spline + solve. */
VLB_API int vlb_poisson(vlb_ctx* ctx, int32_t precision);

/* Precision of the mode products of vlb_coefficients and vlb_mean_field
 * (vlb_poisson and vlb_step set it too).  No counterpart in the reference,
 * whose products are SGEMM on CUDA devices. */
VLB_API int vlb_set_precision(vlb_ctx* ctx, int32_t precision);

/* spline_coefficients!(csol, phi, dm) (src/devicemesh.jl:126-127) into the
 * level's csol grid.  level: 0 fine, 1 coarse. */
VLB_API int vlb_coefficients(vlb_ctx* ctx, int32_t level);

/* effective_potential!(csol, rho, dm, jel) (src/devicemesh.jl:171-183):
 * csol += S^-1 [V_xc(rho) + V_jel(r)]. */
VLB_API int vlb_mean_field(vlb_ctx* ctx, int32_t level, double nions, double radius);

/* forces!(cloud, acc, fine, csolf, coarse, csolc, sm; projectile, packed=true)
 * (src/accelerator.jl:607-733), with the out-of-stencil tail on the device.
 * Uses the csol grids in place.  red[4] receives the projectile sums. */
VLB_API int vlb_forces(vlb_ctx* ctx, const vlb_projectile* proj, double red[4], int32_t* outcount);

/* projectile_forces!(cloud, acc, proj, jel) (src/accelerator.jl:746-756)
 * from the sums of the last vlb_forces. */
VLB_API int vlb_projectile_forces(vlb_ctx* ctx, const vlb_projectile* proj, double nions,
                          double jellium_radius, double force[3], double* e_electrons,
                          double* e_jellium);

/* step!(cloud, dt, acc; rcmax) (src/accelerator.jl:580-605): packed Verlet.
 * diag = kinetic, escaped, angular x, y, z. */
VLB_API int vlb_push(vlb_ctx* ctx, double dt, double rcmax, double diag[5]);

/* step!(sim; energy=false) on the resident path (src/simulation.jl:382-416,
 * 472-531) fused into one stream of kernels with no host synchronisation
 * inside; `proj` is read and updated (the projectile's Verlet step,
 * src/projectile.jl:298-304). */
VLB_API int vlb_step(vlb_ctx* ctx, vlb_projectile* proj, const vlb_step_params* params,
             vlb_step_result* result);

/* ---- the same step sharded over several contexts (one per GPU), each
 * holding a slice of the cloud.  No counterpart in the reference, which runs
 * one device.  The step is the three phases below; between them the caller
 * sums the exchange buffers over the shards, in place, on the context's
 * stream (an all-reduce):
 *   vlb_step_deposit  : sort, raw fine deposit, coarse deposit;
 *                       then sum rho_fine, rho_coarse and scalars;
 *   vlb_step_fields   : renormalise with the whole cloud's count, nested
 *                       Poisson solve, mean field (identical on every shard),
 *                       forces on this shard's particles;
 *                       then sum reaction (the projectile's reaction sums);
 *   vlb_step_advance  : projectile step (identical on every shard), push,
 *                       capture count; results are this shard's (sum the
 *                       kinetic, escaped, angular, enclosed and counts).
 * With the fixed-point deposit the summed densities do not depend on the
 * order of the sum.  One context alone is vlb_step. */
#define VLB_DTYPE_FLOAT32 0
#define VLB_DTYPE_INT64 1

typedef struct vlb_exchange {
  void* rho_fine;             /* n^3 of rho_fine_dtype: the raw fine deposit */
  int32_t rho_fine_dtype;     /* VLB_DTYPE_INT64 (fixed point) or VLB_DTYPE_FLOAT32 */
  int32_t pad0_;
  int64_t rho_fine_count;
  void* rho_coarse;           /* n^3 of rho_coarse_dtype: the coarse deposit */
  int32_t rho_coarse_dtype;   /* VLB_DTYPE_INT64 (fixed point) or VLB_DTYPE_FLOAT32 */
  int32_t pad3_;
  int64_t rho_coarse_count;
  double* scalars;            /* float64: [0] particles outside the deposit window */
  int32_t scalars_count;
  int32_t pad1_;
  double* reaction;           /* float64 [4]: the projectile's reaction sums */
  int32_t reaction_count;
  int32_t pad2_;
  void* stream;               /* the context's cudaStream_t */
} vlb_exchange;

/* ---- the learned denoiser of the fine density.  No counterpart in the
 * reference.  A 3-D convolutional network (four 3^3 layers, 1-16-16-16-3
 * channels, ReLU, no biases; BF16 weights, float32 arithmetic; weights of
 * layer l as [27][cin][cout], tap = dx + 3 dy + 9 dz).  Its three outputs are
 * a charge flux F = f(s rho) and the density it gives is
 * out = rho + div F^ / s, F^ the flux with none through the grid's faces
 * and limited so that no voxel gives more charge than it holds: the network
 * moves charge between neighbouring voxels, adds none and makes no negative
 * density.  It is trained on
 * pairs of densities of the method itself (an 8e6-particle run's deposit
 * against a run with ten times the particles, at the same instant).
 *
 * In the step (vlb_step_params.denoise): after the renormalised fine
 * deposit, the network's density replaces the deposit's when their charges
 * differ by at most charge_tolerance (electrons), renormalised to the
 * deposit's charge; otherwise the deposit stays (vlb_step_result.denoised).
 * The building blocks below (device pointers, the caller's stream) are what
 * a training loop needs: the forward pass, the loss gradient against a
 * target density, an Adam update. */
VLB_API int vlb_dn_weight_count(void);
VLB_API int vlb_set_denoiser(vlb_ctx* ctx, const float* weights, int32_t count, double input_scale,
                     double charge_tolerance);
VLB_API int vlb_clear_denoiser(vlb_ctx* ctx);

typedef struct vlb_denoiser vlb_denoiser;
VLB_API int vlb_dn_create(int32_t nx, int32_t ny, int32_t nz, int32_t device, vlb_denoiser** out);
VLB_API int vlb_dn_destroy(vlb_denoiser* dn);
/* out = x + div f(scale x) / scale over an nx*ny*nz float32 grid (device pointers) */
VLB_API int vlb_dn_forward(vlb_denoiser* dn, const float* x, float scale, const float* weights, float* out,
                   void* stream);
/* grad = d loss / d weights, loss = mean over voxels of (scale (out - target))^2 (host, may be null) */
VLB_API int vlb_dn_gradient(vlb_denoiser* dn, const float* x, const float* target, float scale,
                    const float* weights, float* grad, double* loss, void* stream);
VLB_API int vlb_dn_adam(vlb_denoiser* dn, float* weights, const float* grad, float* m, float* v, float lr,
                int32_t step, void* stream);
/* device flags raised by the denoiser's kernels since the last call (a
 * tensor-core wait that gave up: VLB_STATUS_MMA_TIMEOUT); synchronises */
VLB_API int vlb_dn_status(vlb_denoiser* dn, int32_t* flags);
/* tiles of 8^3 voxels the last pass computed: those within one tile of a
 * tile whose largest |x| exceeds 1e-3 of the volume's (the others pass
 * through unchanged) */
VLB_API int vlb_dn_active_tiles(vlb_denoiser* dn, int32_t* n);

/* ---- the energy budget's sums (interaction_energy, src/energy.jl:19-43):
 * sum over the cloud of w phi(p), phi the smoothed fine potential inside the
 * host margin knots[3] < p < knots[end-2], the coarse spline outside it, 0
 * outside both, for the total coefficients (csol, as after a step) or the
 * Hartree ones (S^-1 phi before the mean field; the fine level's are those
 * of the last step run with params.energy).  The cloud may have moved since
 * its last sort (as after a push).  Synchronises. */
/* ---- the film: the density slices and capture scalars of the reference's
 * movie (scripts/xenon.jl:370-410, which reads sim.rho and the cloud back to
 * the host for every frame and renders them with GLMakie/Cairo), kept on the
 * device as headless buffers.  Rendering is out of scope; the frames go to
 * the caller as arrays.
 *
 * vlb_film_reserve allocates `capacity` frames (and frees any earlier film).
 * A vlb_step with params.film = 1 then appends one frame after its push:
 *   frame f: n*n float32, i fastest, the fine density's plane average
 *            (rho[:, :, iz1] + rho[:, :, iz2]) / 2 in float32 (0-based planes;
 *            the script's reaction plane is iz1 = nfine - 1, iz2 = nfine);
 *   scalars[4 f .. 4 f + 3]: the projectile's x and y after the step, the
 *            particles within params.capture_radius of it (0 when that radius
 *            is <= 0) and the particles within `radius` of the origin (the
 *            script's net charge is nions - weight * that count, radius 35).
 * Frames past the capacity are counted, not stored.  Steps with film = 0 run
 * the film's kernels as no-ops (the captured step keeps them); batch and
 * sharded steps take no frames (they return VLB_ERR_ARG when params.film is
 * set).  Reserving or clearing drops the captured
 * step.  No counterpart entry point in the reference. */
VLB_API int vlb_film_reserve(vlb_ctx* ctx, int32_t capacity, int32_t iz1, int32_t iz2, double radius);
/* Frames asked for since the reservation (taken) and held (stored = min(taken,
 * capacity)).  Synchronises. */
VLB_API int vlb_film_frames(vlb_ctx* ctx, int32_t* taken, int32_t* stored);
/* Frames [first, first + count) to host arrays: frames [count*n*n] float32,
 * scalars [4*count] float64 (either may be NULL).  Synchronises. */
VLB_API int vlb_film_download(vlb_ctx* ctx, int32_t first, int32_t count, float* frames, double* scalars);
VLB_API int vlb_film_clear(vlb_ctx* ctx);

#define VLB_ENERGY_TOTAL 0
#define VLB_ENERGY_HARTREE 1
VLB_API int vlb_interaction_energy(vlb_ctx* ctx, int32_t coefficients, double* out);

/* ---- launch shapes.  No counterpart in the reference (whose kernels take
 * fixed workgroup sizes, src/accelerator.jl:253-259).  chunk: particles per
 * work item of the gather and the coarse deposit (a multiple of 32, 32 to
 * 4096); the others: CTAs per SM of the persistent grids.  Results do not
 * depend on them except for the order of float32 atomic sums.  Setting them
 * drops the captured step; the next step re-sorts. */
typedef struct vlb_tuning {
  int32_t chunk;              /* 128 */
  int32_t field_ctas_per_sm;  /* 3: the smoothed gather */
  int32_t cic_ctas_per_sm;    /* 4: the coarse deposit */
  int32_t push_ctas_per_sm;   /* 2: the Verlet push */
  int32_t move_ctas_per_sm;   /* 4: the record move of the sort */
  int32_t field_tensor_cores; /* 1: the gather's sums over y as 3xTF32 MMAs
                                 (tcgen05, two CTAs per SM, field_ctas_per_sm
                                 unused; needs chunk <= 128); 0: FP32 FMAs */
  int32_t scan_wait_polls;    /* 0: the sort's look-back waits give up after
                                 4,194,304 polls; n > 0: after n; -1: at once
                                 (a test of the bounded waits).  A wait that
                                 gives up sets VLB_STATUS_SCAN_TIMEOUT (the step
                                 returns VLB_ERR_TIMEOUT) and its tile sums its
                                 predecessors' inputs itself: the sort stays
                                 exact. */
  int32_t reserved[1];
} vlb_tuning;

VLB_API int vlb_set_tuning(vlb_ctx* ctx, const vlb_tuning* tuning);
VLB_API int vlb_get_tuning(vlb_ctx* ctx, vlb_tuning* tuning);

/* ---- batches: several independent runs (contexts on one device, e.g. an
 * impact-parameter / projectile sweep with clouds of different sizes)
 * stepped together.  No counterpart in the reference, which runs one
 * collision per process.  vlb_batch_step advances every context by one
 * step (projs[i] and results[i] belong to the i-th context; params are
 * shared), each on its own stream, forked from and joined to the batch's
 * stream; with params->use_graph the whole batch step is captured once as
 * one CUDA graph and replayed.  params->push must be 1 (priming goes
 * through vlb_step). */
typedef struct vlb_batch vlb_batch;
VLB_API int vlb_batch_create(vlb_ctx* const* ctxs, int32_t n, vlb_batch** out);
VLB_API int vlb_batch_step(vlb_batch* batch, vlb_projectile* projs, const vlb_step_params* params,
                   vlb_step_result* results);
VLB_API int vlb_batch_destroy(vlb_batch* batch);

/* Device addresses of the exchange buffers (valid for the context's life). */
VLB_API int vlb_exchange_buffers(vlb_ctx* ctx, int32_t deposit_mode, vlb_exchange* out);
VLB_API int vlb_step_deposit(vlb_ctx* ctx, const vlb_projectile* proj, const vlb_step_params* params);
/* npart_global: particles in all shards together. */
VLB_API int vlb_step_fields(vlb_ctx* ctx, const vlb_step_params* params, int64_t npart_global);
VLB_API int vlb_step_advance(vlb_ctx* ctx, vlb_projectile* proj, const vlb_step_params* params,
                     vlb_step_result* result);

/* sync_host! (src/simulation.jl:544-552) for one grid, and its inverse. */
VLB_API int vlb_get_grid(vlb_ctx* ctx, int32_t which, float* host);
VLB_API int vlb_set_grid(vlb_ctx* ctx, int32_t which, const float* host);

/* The force buffer acc.force, SoA 3*npart, in slot order. */
VLB_API int vlb_get_forces(vlb_ctx* ctx, float* host);
/* The forces of slots [first, first + count): host SoA [3*count]. */
VLB_API int vlb_get_forces_range(vlb_ctx* ctx, int64_t first, int64_t count, float* host);
VLB_API int vlb_set_forces(vlb_ctx* ctx, const float* host);

/* enclosed_charge(cloud, proj, radius) (src/projectile.jl:243-247) on the
 * device-resident cloud. */
VLB_API int vlb_enclosed_charge(vlb_ctx* ctx, const double position[3], double radius, double* q);

/* Accumulated device time per stage since the last reset (ms), measured
 * with CUDA events when profiling is on; names via vlb_stage_name.  Stages
 * 0..8 tile the step (sort .. capture); stage 10, "forces_kernel", is the
 * gather kernel alone, inside stage 5; stage 9 is unused. */
VLB_API int vlb_profile(vlb_ctx* ctx, int32_t enable);
VLB_API int vlb_stage_count(void);
VLB_API const char* vlb_stage_name(int32_t i);
VLB_API int vlb_stage_times(vlb_ctx* ctx, double* ms, int32_t n);
/* Kernel launches issued by this context so far. */
VLB_API int vlb_launch_count(vlb_ctx* ctx, int64_t* count);
/* FP32 FMA throughput of the device at its current clocks (TFLOP/s), the
 * ceiling the FP32-bound kernels (gather, fine deposit) are measured against.
 * No counterpart in the reference: a measurement helper. */
VLB_API int vlb_fp32_peak(int32_t device, double* tflops);
/* The context's CUDA stream (cudaStream_t), for event timing by a caller. */
VLB_API int vlb_stream(vlb_ctx* ctx, void** stream);

/* Total charge sum_ijk rho[i,j,k] m0[i] m0[j] m0[k] of a density the caller
 * holds on the device, for callers that cannot allocate device memory: an
 * embedding runtime whose caching pool has already claimed the GPU's memory;
 * a plugin whose host forbids allocation outside its set-up phase; a loop
 * that must not stall on cudaMalloc's synchronisation.  It allocates nothing:
 * the scratch (one float64 per (j,k) column) is a fixed 512 KiB of static
 * device memory that every GPU loading the library keeps until exit, so n is
 * at most 256 points per axis; larger n returns VLB_ERR_ARG.
 * rho: device float32 [n*n*n], i fastest; m0: device float64 [n] (order-0 dual
 * moments); q: device float64 [1], written; stream: a cudaStream_t, or NULL.
 * Runs on the current device.  The first call on a device resolves the
 * scratch's device address and caches it for the rest of the process; make
 * it before any stream capture.  The cache assumes the device's context lives
 * until exit: resetting the device (cudaDeviceReset) or tearing down and
 * recreating its primary context between calls is not supported.  Calls share
 * the scratch: calls that overlap on the GPU race, so keep them on one stream.
 * No counterpart in the reference (its total_charge allocates through its
 * backend); the reduction is the one vlb_deposit_fine applies. */
VLB_API int vlb_total_charge_noalloc(const float* rho, const double* m0, int32_t n, double* q, void* stream);

/* ---- host-side set-up helpers (no GPU needed) ---- */

/* sample_thomas_fermi(profile::RadialProfile, npart, weight; rng = Ran2(seed))
 * (src/initial.jl:184-203) with the thesis's ran2 (src/random.jl:31-90;
 * consistent != 0 restores IQ1 = 53668).  positions, momenta: AoS 3*npart. */
VLB_API int vlb_sample_thomas_fermi(const double* quantiles, int32_t nq, const double* density,
                            int32_t nrho, double rmax, int64_t npart, double weight,
                            int32_t seed, int32_t consistent, double* positions,
                            double* momenta);

/* The same draw as a stream (the construction of src/initial.jl:94-113 a
 * chunk at a time): vlb_sampler_draw(s, n, ...) returns the next n particles
 * of the Ran2(seed) cloud, so consecutive draws give the one-shot cloud bit
 * for bit.  positions = momenta = NULL skips n particles (their uniforms are
 * still consumed), as a rank that keeps only its slice of the cloud does.
 * The sampler keeps copies of the profile tables. */
typedef struct vlb_sampler vlb_sampler;
VLB_API int vlb_sampler_create(const double* quantiles, int32_t nq, const double* density, int32_t nrho,
                       double rmax, double weight, int32_t seed, int32_t consistent, vlb_sampler** out);
VLB_API int vlb_sampler_draw(vlb_sampler* sampler, int64_t n, double* positions, double* momenta);
VLB_API int vlb_sampler_destroy(vlb_sampler* sampler);

/* next!(Ran2(seed)) n times (src/random.jl:80-90). */
VLB_API int vlb_ran2(int32_t seed, int32_t consistent, int64_t n, float* out);

/* PackedPositions setindex! split (src/particles.jl:135-149): positions AoS
 * 3*npart -> knode, delta SoA 3*npart; and the inverse getindex
 * (src/particles.jl:128-132). */
VLB_API int vlb_pack_positions(int64_t npart, const double* positions, double x0, double h,
                       int32_t* knode, float* delta);
VLB_API int vlb_unpack_positions(int64_t npart, const int32_t* knode, const float* delta,
                         double x0, double h, double* positions);

#ifdef __cplusplus
}
#endif

#endif /* VLASOV_B200_H */
