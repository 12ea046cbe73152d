// Internal declarations of the B200 library: the context, the device scalar
// block, and the launch wrappers each kernel file exports.
#pragma once

#include <cuda.h>  // CUtensorMap and its enums (the encoder is reached through the runtime)
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vlasov_b200.h"

namespace vlb {

constexpr int kWarp = 32;
constexpr int kNumStages = 12;
// Events 10 and 11 of a profiled step bracket the gather kernel alone; its
// time is stage 10 ("forces_kernel").
constexpr int kEvGatherBegin = 10;
constexpr int kEvGatherEnd = 11;
constexpr int kChunk = 128;       // default particles per work item of the gather and CIC
constexpr int kMinChunk = 32;     // smallest chunk a tuning may set (sizes the item list)

// Error flags raised by kernels into DeviceScalars::status.
constexpr int kStatusScanTimeout = VLB_STATUS_SCAN_TIMEOUT;  // decoupled look-back gave up
constexpr int kStatusBadCell = VLB_STATUS_BAD_CELL;          // a particle outside the CIC domain table
constexpr int kStatusOverflow = VLB_STATUS_OVERFLOW;         // fixed-point accumulator out of range
constexpr int kStatusMmaTimeout = VLB_STATUS_MMA_TIMEOUT;    // a tensor-core kernel gave up waiting

// A matrix split into head and tail for the tensor-core mode products, in
// the canonical K-major no-swizzle layout: [hi | lo] in TF32 (img, each
// npad16 x kpad8 floats) and in BF16 (bimg, each npad16 x kpad16 halves).
struct TcImage {
  float* img = nullptr;
  uint16_t* bimg = nullptr;
  int n = 0, npad16 = 0, kpad8 = 0, kpad16 = 0;
};

// Device-resident scalars of one step.  One block, zeroed (partly) at the
// start of a step and copied back in one transfer at its end.
struct DeviceScalars {
  // --- reset every step (everything up to `reset_end`) ---
  unsigned long long work_deposit;   // dynamic work counters
  unsigned long long work_gather;
  unsigned long long scan_tiles[8];  // tile tickets of the look-back scans
  int32_t nout;                      // deposit window rejections
  int32_t outcount;                  // out-of-stencil slots
  int32_t noccupied;
  int32_t status;
  double red[4];                     // projectile sums (gaussian kernel)
  double diag[5];                    // kinetic, escaped, angular xyz
  double moments[10];                // multipole sums (coarse)
  double charge_raw;                 // fine charge before renormalisation
  unsigned long long enclosed;       // particles within the capture radius
  unsigned long long work_cic;
  int32_t nitems;                    // cell chunks of the gather
  int32_t pad_items;
  double xch[4];                     // exchanged between the shards of a step: [0] deposit-window rejections;
                                     // [1] charge of the denoiser's prediction (not exchanged)
  int32_t denoised;                  // 1: the step used the denoiser's density
  int32_t pad_dn;
  unsigned long long work_energy;    // work counter of the energy kernel
  double energy[2];                  // sum w phi: [0] on the Hartree coefficients, [1] on the total
  int32_t sort_far;                  // the nearly sorted path of the sort gave up (1: a far mover, 2: a count)
  int32_t reset_end;
  // --- persistent ---
  double multipole[10];              // q, centre xyz, quadrupole (xx yy zz xy xz yz)
  double proj_pos[3], proj_prev[3], proj_vel[3], proj_force[3];
  double proj_charge, proj_mass, proj_sigma, proj_ball;
  int32_t proj_active;
  int32_t proj_soft;                 // VLB_SOFTENING_DEVICE or VLB_SOFTENING_BALL
  int32_t film_due;                  // 1: this step appends a film frame (uploaded with the projectile)
  int32_t pad_film;
  double e_el, e_jel;
  unsigned long long film_inside;    // particles within the film radius of the origin (a frame's count)
  int32_t film_next;                 // frames taken since vlb_film_reserve
  int32_t film_pad;
  int32_t nocc_par[2];               // occupied cells of the sort products of each parity
  int32_t nitems_par[2];             // and their work items
};

struct Level {
  int nk = 0, n = 0, ni = 0;        // knots, points, interior points per axis
  int npad = 0, nipad = 0;          // padded row counts of the transposed matrices
  // float32 tables
  float* colloc = nullptr;          // [n]
  float* knots = nullptr;           // [nk]
  float* sinvT = nullptr;           // [n][npad]  (S^-1)^T, zero padded
  float* MT = nullptr;              // [ni][nipad]
  float* MinvT = nullptr;           // [ni][nipad]
  TcImage tc_sinv, tc_M, tc_Minv;   // the same matrices for the 3xTF32 products
  float* lap = nullptr;             // [n*n] row-major
  float* invlsum = nullptr;         // [ni^3]
  float* dual = nullptr;            // [3n]
  float* dlen = nullptr;            // [n]
  double* dual_d = nullptr;         // [3n] float64 copy for the reductions
  double* knots_d = nullptr;        // [nk] float64 copy for the host-tail field
  int32_t* loc_cells = nullptr;     // [loc_ncell]
  int loc_ncell = 0;
  float loc_x0 = 0, loc_invw = 0;
  // grids
  float* rho = nullptr;
  float* phi = nullptr;
  float* csol = nullptr;
  float* csol_hartree = nullptr;    // S^-1 phi before the mean field (coarse: every step; fine: energy steps)
  // host copies kept for reference
  std::vector<double> h_knots, h_colloc;
};

struct Particles {
  int32_t* k = nullptr;   // [3*Npad]
  float* d = nullptr;
  int32_t* pk = nullptr;
  float* pd = nullptr;
};

struct Denoiser;

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  int64_t N = 0, Npad = 0;
  double weight = 0;
  Level fine, coarse;
  // fine-axis constants as the reference's kernels see them (Float32)
  double x0 = 0, h = 0;
  float x0f = 0, hf = 0, spacing_f = 0, lo_f = 0, hi_f = 0;
  int nbdt = 0, ncol = 0;
  float* overlap = nullptr;   // [ncol][10]
  float* gradient = nullptr;  // [ncol][10]
  float* ovgr = nullptr;      // [ncol][20]: each column's overlap row, then its gradient row (80-byte rows)
  float* nodes = nullptr;     // [ncol][8]
  // particle state, double buffered for the sort
  Particles part[2];
  int cur = 0;
  float* force = nullptr;     // [3*Npad] SoA
  // sort
  int ncell = 0;
  uint32_t* keys = nullptr;      // [N] unsorted cell keys
  uint32_t* keys_alt = nullptr;  // [N]
  uint32_t* skeys = nullptr;     // [N] sorted cell keys (slot order)
  uint32_t* perm = nullptr;      // [N]
  // [N] each slot's fine-deposit table columns (10 bits each, minus one) and
  // bit 30 set outside the deposit window, written by the sort's record move
  // when ncol <= 1024 (cols_packed)
  uint32_t* cols = nullptr;
  bool cols_packed = false;
  uint32_t* vals_alt = nullptr;  // [N]
  uint32_t* radix_table = nullptr;
  int64_t radix_table_size = 0;
  int32_t* counts = nullptr;     // [ncell]
  int32_t* cell_off = nullptr;   // [ncell]
  // The sort's products by parity: buffers p describe part[p]'s slot order
  // after the sort that filled part[p].  occupied and bounds point at the
  // current parity's.
  int32_t* occ_buf[2] = {nullptr, nullptr};   // [ncell] occupied cells, increasing
  int32_t* bnd_buf[2] = {nullptr, nullptr};   // [ncell+1]
  int32_t* cidx_buf[2] = {nullptr, nullptr};  // [ncell] cell -> its index in occ_buf (occupied cells only)
  int32_t* occupied = nullptr;
  int32_t* bounds = nullptr;
  int32_t* dir_cnt = nullptr;    // [min(ncell, N)][27] nearly sorted path: particles per (old cell, direction)
  int32_t* dir_base = nullptr;   // [min(ncell, N)][27] their first slot in the new order
  bool order_valid = false;      // part[cur] is in the order its sort products describe
  bool last_sort_near = false;   // the last sort tried the nearly sorted path
  bool graph_sort_near = false;  // the captured step graphs' sorts try it
  bool prev_deferred = false;    // the last sort left (pk, pdelta) in part[cur ^ 1], in the
                                // order before it: its push (or settle_prev) moves them
  int32_t* outlist = nullptr;    // [N]
  int32_t* chunk_start = nullptr;  // [ncell] first chunk of occupied cell g (current parity's)
  int32_t* item_cell = nullptr;    // [N / kMinChunk + ncell] occupied cell of each chunk (current parity's)
  int4* item_rec = nullptr;        // [N / kMinChunk + ncell] each chunk's cell code, slots and packed knots
                                   // (current parity's)
  int4* rec_buf[2] = {nullptr, nullptr};
  int32_t* cstart_buf[2] = {nullptr, nullptr};
  int32_t* item_buf[2] = {nullptr, nullptr};
  int chunk_par[2] = {kChunk, kChunk};  // the chunk each parity's work items were cut with
  int32_t* item_dir = nullptr;     // [N / kMinChunk + ncell][27] nearly sorted path: per item and direction
  unsigned long long* scan_status = nullptr;  // look-back tile states
  int64_t scan_status_size = 0;
  // deposit
  unsigned long long* rho_fixed = nullptr;    // [n^3] int64 accumulator
  unsigned long long* rho_fixed_c = nullptr;  // [nc^3] the coarse deposit's, in fixed point
  // order-fixed reductions: the projectile's reaction sums per work item of
  // the gather and per CTA of the tail, the push's diagnostics per CTA
  double* red_items = nullptr;                // [max items][4]
  double* red_tail = nullptr;                 // [num_sms][4]
  double* red_blocks = nullptr;               // [num_sms][4] first level of their sum
  double* e_items = nullptr;                  // [max items] interaction energy per work item
  double* e_blocks = nullptr;                 // [num_sms] first level of their sum
  bool items_valid = false;                   // the work items describe the cloud (its last sort)
  double* diag_part = nullptr;                // [num_sms * 32][5]
  double* partials = nullptr;                 // [10 * n^2] reductions
  // Poisson work buffers (max n^3)
  float* work[3] = {nullptr, nullptr, nullptr};
  int mode_precision = 0;     // VLB_POISSON_FP32, VLB_POISSON_3XTF32 or VLB_POISSON_BF16X3
  // launch shapes (vlb_set_tuning): particles per work item, persistent-grid
  // CTAs per SM of the gather, the coarse deposit, the push and the record move
  int chunk = kChunk, field_cps = 3, cic_cps = 4, push_cps = 2, move_cps = 4;
  // polls of a look-back wait before it gives up: 0 the default, -1 none
  // (every tile after the first takes the scan's fallback at once)
  int scan_wait_polls = 0;
  bool field_tc = true;  // the gather's y sums on the tensor cores (chunk <= 128)
  // The fine spline coefficients with rows padded to a multiple of four
  // floats (a pitch of 16-byte multiples), refreshed before each tensor-core
  // gather, and the 3-D tiled tensor map over it from which the gather's
  // stencil tiles are copied by the TMA unit.
  float* csol_rows = nullptr;
  int csol_pitch = 0;
  CUtensorMap csol_map{};
  unsigned* tc_sync = nullptr;  // grid-barrier counter of the tensor-core chains
  // the learned denoiser of the fine density (vlb_set_denoiser)
  Denoiser* dn = nullptr;
  float* dn_weights = nullptr;  // BF16-rounded weights on the device
  float* dn_pred = nullptr;     // [n^3] its prediction
  double dn_scale = 1, dn_tol = 1e-3;
  // the film (vlb_film_reserve): density slices and their scalars
  int film_cap = 0, film_iz1 = 0, film_iz2 = 0;
  double film_r2 = 0;
  float* film_frames = nullptr;    // [film_cap][n_fine^2]
  double* film_scalars = nullptr;  // [film_cap][4]
  // scalars
  DeviceScalars* dsc = nullptr;
  DeviceScalars* hsc = nullptr;  // pinned, results
  DeviceScalars* hin = nullptr;  // pinned, projectile staging
  // state
  bool sorted = false, have_forces = false;
  // keys[] and counts[] hold the cell keys and histogram of part[cur] in slot
  // order (written by the push of a fused step): the next sort skips them
  bool keys_ready = false;
  int shard_phase = 0;  // phases of a sharded step done: 1 deposit, 2 fields
  // profiling
  bool profile = false;
  cudaEvent_t ev[kNumStages + 1];
  bool evs_made = false;
  double stage_ms[kNumStages] = {0};
  long long launches = 0;
  // graphs of the fused step, one per parity of the sort's double buffer
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  vlb_step_params graph_params{};
  bool graph_valid = false;
  uint64_t config_epoch = 0;         // bumped by every change a captured graph bakes in (shapes, denoiser)
  long long graph_launches = 0;  // kernels in one captured step
};

std::string cuda_msg(cudaError_t e, const char* what);
void set_last_error(const std::string& msg);
int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

// ---------------------------------------------------------------- kernels
// sort.cu
// defer_prev: a push follows in the same step and reads the previous
// positions through the permutation, so the move leaves them in place.
void launch_sort(Ctx& c, bool defer_prev = false);
void settle_prev(Ctx& c);
// deposit.cu
void launch_deposit_fine(Ctx& c, double charge, int mode);
void launch_deposit_fine_raw(Ctx& c, int mode);
void launch_deposit_fine_normalize(Ctx& c, double charge, int mode, int64_t npart_global);
void launch_deposit_coarse(Ctx& c, double charge, int mode);
void launch_deposit_coarse_finish(Ctx& c, int mode);
// poisson.cu
void launch_poisson(Ctx& c);
void launch_grid_charge(Ctx& c, Level& L, const float* rho, double* out);
// denoise.cu
Denoiser* dn_create(int nx, int ny, int nz, int device, int num_sms);
void dn_free(Denoiser* d);
void dn_route_status(Denoiser* d, int32_t* status);
void launch_denoise(Ctx& c, int64_t npart_global);
void free_denoiser(Ctx& c);
// mode_tc.cu
bool tc_supported(int n);
TcImage make_tc_image(const double* A, int n);
void tc_setup(Ctx& c);
void launch_mode_chain_tc(Ctx& c, const TcImage& A, int nst, const float* const* src, float* const* dest,
                          const int* epi, long long m, const float* invl);
void launch_coefficients(Ctx& c, Level& L, const float* src, float* dst);
void launch_mean_field_coefficients(Ctx& c, Level& L, const float* phi, float* csol,
                                    double nions, double radius);
void launch_mean_field_add(Ctx& c, Level& L, double nions, double radius);
// gather.cu
void launch_forces(Ctx& c);
void launch_energy(Ctx& c, const float* csolf, const float* csolc, double* out);
// push.cu
void launch_projectile_update(Ctx& c, double dt, double nions, double jradius, int advance);
void launch_projectile_force_only(Ctx& c, double nions, double jradius);
void launch_push(Ctx& c, double dt, double rcmax, double capture_radius, bool keys);
void launch_enclosed(Ctx& c, double radius);
void launch_film(Ctx& c, double capture_radius);


}  // namespace vlb

// Count and check a launch.
#define VLB_LAUNCHED(c)                                                  \
  do {                                                                   \
    (c).launches++;                                                      \
    cudaError_t _e = cudaGetLastError();                                 \
    if (_e != cudaSuccess) throw vlb::CudaError(_e, __FILE__, __LINE__); \
  } while (0)

namespace vlb {
struct CudaError {
  cudaError_t err;
  const char* file;
  int line;
  CudaError(cudaError_t e, const char* f, int l) : err(e), file(f), line(l) {}
};
struct ArgError {
  std::string msg;
  explicit ArgError(std::string m) : msg(std::move(m)) {}
};
}  // namespace vlb

#define VLB_CUDA(x)                                                   \
  do {                                                                \
    cudaError_t _e = (x);                                             \
    if (_e != cudaSuccess) throw vlb::CudaError(_e, __FILE__, __LINE__); \
  } while (0)

// ------------------------------------------------------ device helpers
// IEEE single-precision operations without contraction: the reference's
// kernels compute their discrete choices (columns, cells, Verlet updates)
// with separately rounded Float32 operations.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// table column of an offset (src/kernels.jl:414-419, 770-772)
__device__ __forceinline__ int table_column(float d, float spacing, int nbdt, int ncol) {
  float half = fmul(spacing, 0.5f);
  float v = fadd(fmul(fdiv(fadd(d, half), spacing), (float)nbdt), 0.5f);
  int c = (int)floorf(v) + 1;
  return min(max(c, 1), ncol);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// The fine deposit's table columns and window test of one particle
// (src/kernels.jl:754-779), packed: column - 1 in 10 bits per axis (ncol <=
// 1024) and bit 30 set when the particle lies outside the window (the
// deposit then takes column 1 on every axis, as the reference does).
constexpr uint32_t kColsOutside = 1u << 30;
__device__ __forceinline__ uint32_t deposit_cols(int k0, int k1, int k2, float d0, float d1, float d2, float x0,
                                                 float h, float lo, float hi, float spacing, int nbdt, int ncol) {
  const int kk[3] = {k0, k1, k2};
  const float dd[3] = {d0, d1, d2};
  bool inside = true;
  uint32_t packed = 0;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const float p = fadd(fadd(x0, fmul((float)(kk[ax] - 1), h)), dd[ax]);
    inside = inside && (lo <= p) && (p <= hi);
    packed |= (uint32_t)(table_column(dd[ax], spacing, nbdt, ncol) - 1) << (10 * ax);
  }
  return inside ? packed : (packed | kColsOutside);
}

// 0-based cell of a clamped knot triple
__device__ __forceinline__ uint32_t cell_key(int kx, int ky, int kz, int nk) {
  kx = clampi(kx, 1, nk);
  ky = clampi(ky, 1, nk);
  kz = clampi(kz, 1, nk);
  return (uint32_t)((kx - 1) + nk * ((ky - 1) + nk * (kz - 1)));
}

__device__ __forceinline__ void cell_knots(uint32_t cell, int nk, int& kx, int& ky, int& kz) {
  kx = (int)(cell % nk) + 1;
  cell /= nk;
  ky = (int)(cell % nk) + 1;
  kz = (int)(cell / nk) + 1;
}

// 10^3 stencil of the field fits (src/kernels.jl:375-377)
__device__ __forceinline__ bool field_fits(int kx, int ky, int kz, int n) {
  int bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
  return bx >= 1 && by >= 1 && bz >= 1 && bx + 9 <= n && by + 9 <= n && bz + 9 <= n;
}
// 8^3 stencil of the deposit fits (src/kernels.jl:106-117)
__device__ __forceinline__ bool deposit_fits(int kx, int ky, int kz, int n) {
  int bx = 2 * kx - 5, by = 2 * ky - 5, bz = 2 * kz - 5;
  return bx >= 0 && by >= 0 && bz >= 0 && bx + 8 <= n && by + 8 <= n && bz + 8 <= n;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
