// The C ABI of the library (include/vlasov_b200.h): context set-up, the
// reference-facing calls, and the fused step with its CUDA-graph replay.

#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <new>

#include "vlb_internal.cuh"

namespace vlb {

void deposit_setup(Ctx& c);
void field_setup(Ctx& c);
double measure_fp32_peak(int device);
int grid_for(const Ctx& c, int64_t n, int threads, int per_sm);

namespace {

thread_local std::string g_err;

const char* kStageNames[kNumStages] = {"sort",          "deposit_fine", "deposit_coarse", "poisson",
                                        "coefficients",  "forces",       "projectile",     "push",
                                        "capture",       "unused9",      "forces_kernel",  "reserved11"};

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    char buf[512];
    snprintf(buf, sizeof buf, "CUDA error %d (%s) at %s:%d", (int)e.err, cudaGetErrorString(e.err), e.file, e.line);
    return fail(VLB_ERR_CUDA, buf);
  } catch (const ArgError& e) {
    return fail(VLB_ERR_ARG, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(VLB_ERR_NOMEM, "host allocation failed");
  }
}

template <class T>
T* dalloc(size_t count) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) throw CudaError(e, __FILE__, __LINE__);
  return static_cast<T*>(p);
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

std::vector<float> to_float(const double* src, size_t n) {
  std::vector<float> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = (float)src[i];
  return v;
}

template <class T>
T* upload(const T* host, size_t n) {
  T* d = dalloc<T>(n);
  VLB_CUDA(cudaMemcpy(d, host, n * sizeof(T), cudaMemcpyHostToDevice));
  return d;
}

float* upload_f(const double* src, size_t n) {
  std::vector<float> v = to_float(src, n);
  return upload(v.data(), n);
}

// A^T zero-padded to `pad` columns: out[i][r] = A[r][i]
float* upload_transposed(const double* A, int n, int pad) {
  std::vector<float> v((size_t)n * pad, 0.f);
  for (int r = 0; r < n; ++r)
    for (int i = 0; i < n; ++i) v[(size_t)i * pad + r] = (float)A[(size_t)r * n + i];
  return upload(v.data(), v.size());
}

void check_level(const vlb_level_desc& L, const char* name) {
  if (L.nknots < 6) throw ArgError(std::string(name) + ": at least 6 knots are required");
  if (!L.knots || !L.colloc || !L.sinv || !L.laplacian || !L.eigvec || !L.eigvec_inv || !L.eigval ||
      !L.dual_moments || !L.dual_lengths || !L.locate_cells || L.locate_ncells < 1)
    throw ArgError(std::string(name) + ": a table pointer is null");
  for (int i = 1; i < L.nknots; ++i)
    if (!(L.knots[i] > L.knots[i - 1])) throw ArgError(std::string(name) + ": knots must increase");
}

void setup_level(Level& D, const vlb_level_desc& L, bool coarse) {
  D.nk = L.nknots;
  D.n = 2 * L.nknots;
  D.ni = D.n - 2;
  D.npad = (D.n + 7) / 8 * 8;
  D.nipad = (D.ni + 7) / 8 * 8;
  if (D.npad > 256) throw ArgError("at most 128 knots per axis are supported");
  const int n = D.n, ni = D.ni;
  D.h_knots.assign(L.knots, L.knots + D.nk);
  D.h_colloc.assign(L.colloc, L.colloc + n);
  D.colloc = upload_f(L.colloc, n);
  D.knots = upload_f(L.knots, D.nk);
  D.knots_d = upload(L.knots, D.nk);
  D.sinvT = upload_transposed(L.sinv, n, D.npad);
  D.MT = upload_transposed(L.eigvec, ni, D.nipad);
  D.MinvT = upload_transposed(L.eigvec_inv, ni, D.nipad);
  D.tc_sinv = make_tc_image(L.sinv, n);
  D.tc_M = make_tc_image(L.eigvec, ni);
  D.tc_Minv = make_tc_image(L.eigvec_inv, ni);
  D.lap = upload_f(L.laplacian, (size_t)n * n);
  {
    std::vector<float> il((size_t)ni * ni * ni);
    const double* lam = L.eigval;
    for (int k = 0; k < ni; ++k)
      for (int j = 0; j < ni; ++j)
        for (int i = 0; i < ni; ++i) {
          const double s = (lam[i] + lam[j]) + lam[k];
          if (s == 0.0) throw ArgError("eigenvalue sum vanishes: singular operator");
          il[(size_t)i + (size_t)ni * (j + (size_t)ni * k)] = (float)(1.0 / s);
        }
    D.invlsum = upload(il.data(), il.size());
  }
  D.dual = upload_f(L.dual_moments, 3 * (size_t)n);
  D.dual_d = upload(L.dual_moments, 3 * (size_t)n);
  D.dlen = upload_f(L.dual_lengths, n);
  D.loc_cells = upload(L.locate_cells, L.locate_ncells);
  D.loc_ncell = L.locate_ncells;
  D.loc_x0 = (float)L.locate_x0;
  D.loc_invw = (float)L.locate_invwidth;
  const size_t tot = (size_t)n * n * n;
  D.rho = dalloc<float>(tot);
  D.phi = dalloc<float>(tot);
  D.csol = dalloc<float>(tot);
  VLB_CUDA(cudaMemset(D.rho, 0, tot * sizeof(float)));
  VLB_CUDA(cudaMemset(D.phi, 0, tot * sizeof(float)));
  VLB_CUDA(cudaMemset(D.csol, 0, tot * sizeof(float)));
  D.csol_hartree = dalloc<float>(tot);
  VLB_CUDA(cudaMemset(D.csol_hartree, 0, tot * sizeof(float)));
}

void free_level(Level& D) {
  dfree(D.colloc); dfree(D.knots); dfree(D.knots_d); dfree(D.sinvT); dfree(D.MT); dfree(D.MinvT);
  dfree(D.tc_sinv.img); dfree(D.tc_M.img); dfree(D.tc_Minv.img);
  dfree(D.tc_sinv.bimg); dfree(D.tc_M.bimg); dfree(D.tc_Minv.bimg);
  dfree(D.lap); dfree(D.invlsum); dfree(D.dual); dfree(D.dual_d); dfree(D.dlen); dfree(D.loc_cells);
  dfree(D.rho); dfree(D.phi); dfree(D.csol); dfree(D.csol_hartree);
}

void destroy_ctx(Ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int g = 0; g < 2; ++g) {
    if (c->gexec[g]) cudaGraphExecDestroy(c->gexec[g]);
    c->gexec[g] = nullptr;
  }
  free_level(c->fine);
  free_level(c->coarse);
  dfree(c->overlap); dfree(c->gradient); dfree(c->ovgr); dfree(c->nodes);
  for (int b = 0; b < 2; ++b) {
    dfree(c->part[b].k); dfree(c->part[b].d); dfree(c->part[b].pk); dfree(c->part[b].pd);
  }
  dfree(c->force);
  dfree(c->csol_rows);
  dfree(c->keys); dfree(c->keys_alt); dfree(c->skeys); dfree(c->perm); dfree(c->cols); dfree(c->vals_alt);
  dfree(c->radix_table); dfree(c->counts); dfree(c->cell_off);
  for (int p = 0; p < 2; ++p) { dfree(c->occ_buf[p]); dfree(c->bnd_buf[p]); dfree(c->cidx_buf[p]); }
  dfree(c->dir_cnt); dfree(c->dir_base);
  dfree(c->outlist);
  for (int p = 0; p < 2; ++p) { dfree(c->cstart_buf[p]); dfree(c->item_buf[p]); dfree(c->rec_buf[p]); }
  dfree(c->item_dir); dfree(c->scan_status); dfree(c->rho_fixed); dfree(c->partials);
  dfree(c->rho_fixed_c); dfree(c->red_items); dfree(c->red_tail); dfree(c->red_blocks); dfree(c->diag_part);
  dfree(c->e_items); dfree(c->e_blocks);
  for (auto& w : c->work) dfree(w);
  free_denoiser(*c);
  dfree(c->film_frames);
  dfree(c->film_scalars);
  dfree(c->tc_sync);
  dfree(c->dsc);
  if (c->hsc) cudaFreeHost(c->hsc);
  if (c->hin) cudaFreeHost(c->hin);
  if (c->evs_made)
    for (auto& e : c->ev) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

Level& level_of(Ctx& c, int level) {
  if (level == 0) return c.fine;
  if (level == 1) return c.coarse;
  throw ArgError("level must be 0 (fine) or 1 (coarse)");
}

float* grid_ptr(Ctx& c, int which) {
  switch (which) {
    case VLB_GRID_RHO_FINE: return c.fine.rho;
    case VLB_GRID_RHO_COARSE: return c.coarse.rho;
    case VLB_GRID_PHI_FINE: return c.fine.phi;
    case VLB_GRID_PHI_COARSE: return c.coarse.phi;
    case VLB_GRID_CSOL_FINE: return c.fine.csol;
    case VLB_GRID_CSOL_COARSE: return c.coarse.csol;
    case VLB_GRID_CSOL_HARTREE_FINE: return c.fine.csol_hartree;
    case VLB_GRID_CSOL_HARTREE_COARSE: return c.coarse.csol_hartree;
    default: throw ArgError("unknown grid selector");
  }
}

size_t grid_size(Ctx& c, int which) {
  const Level& L = (which % 2 == 0) ? c.fine : c.coarse;
  return (size_t)L.n * L.n * L.n;
}

// projectile -> device scalars (persistent part)
void upload_projectile(Ctx& c, const vlb_projectile* p, int32_t film_due = 0) {
  DeviceScalars& h = *c.hin;
  h.film_due = film_due;
  for (int d = 0; d < 3; ++d) {
    h.proj_pos[d] = p ? p->position[d] : 0.0;
    h.proj_prev[d] = p ? p->previous[d] : 0.0;
    h.proj_vel[d] = p ? p->velocity[d] : 0.0;
    h.proj_force[d] = 0.0;
  }
  h.proj_charge = p ? p->charge : 0.0;
  h.proj_mass = p ? p->mass : 1.0;
  h.proj_sigma = p ? p->sigma : 1.0;
  h.proj_ball = p ? p->ball_radius : 1.0;
  h.proj_active = p ? p->active : 0;
  if (p && p->softening != VLB_SOFTENING_DEVICE && p->softening != VLB_SOFTENING_BALL)
    throw ArgError("projectile softening must be VLB_SOFTENING_DEVICE or VLB_SOFTENING_BALL");
  h.proj_soft = p ? p->softening : VLB_SOFTENING_DEVICE;
  const size_t off = offsetof(DeviceScalars, proj_pos);
  const size_t len = offsetof(DeviceScalars, film_due) + sizeof(int32_t) - off;
  VLB_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(c.dsc) + off, reinterpret_cast<char*>(c.hin) + off, len,
                           cudaMemcpyHostToDevice, c.stream));
}

void fetch_scalars(Ctx& c) {
  VLB_CUDA(cudaMemcpyAsync(c.hsc, c.dsc, sizeof(DeviceScalars), cudaMemcpyDeviceToHost, c.stream));
  VLB_CUDA(cudaStreamSynchronize(c.stream));
}

int status_code(Ctx& c) {
  int s = c.hsc->status;
  if (s & kStatusScanTimeout) return fail(VLB_ERR_TIMEOUT, "a device scan gave up waiting on a predecessor tile");
  if (s & kStatusMmaTimeout)
    return fail(VLB_ERR_TIMEOUT, "a tensor-core mode product gave up waiting on its copies or MMAs");
  if (s) return fail(VLB_ERR_STATE, "device status flags set: " + std::to_string(s));
  return VLB_OK;
}

void stage_mark(Ctx& c, int i) {
  if (c.profile) VLB_CUDA(cudaEventRecord(c.ev[i], c.stream));
}

// occupied / bounds name the sort products that describe part[cur]
void sync_sort_products(Ctx& c) {
  c.occupied = c.occ_buf[c.cur];
  c.bounds = c.bnd_buf[c.cur];
  c.item_cell = c.item_buf[c.cur];
  c.item_rec = c.rec_buf[c.cur];
  c.chunk_start = c.cstart_buf[c.cur];
}

void reset_step_scalars(Ctx& c) {
  VLB_CUDA(cudaMemsetAsync(c.dsc, 0, offsetof(DeviceScalars, reset_end), c.stream));
}

// The fused step: everything on the stream, no host synchronisation.
// Stage events are recorded only when profiling (never inside a capture).
// It runs in three phases; a sharded step exchanges between them (the raw
// deposits and the deposit-window count after the first, the projectile's
// reaction sums after the second).  normalize_npart > 0: renormalise the
// fine density inside the phase (the whole cloud is in this context).
void enqueue_phase_deposit(Ctx& c, const vlb_step_params& p, int64_t normalize_npart) {
  reset_step_scalars(c);
  stage_mark(c, 0);
  launch_sort(c, p.push != 0);
  stage_mark(c, 1);
  launch_deposit_fine_raw(c, p.deposit_mode);
  if (normalize_npart > 0) {
    launch_deposit_fine_normalize(c, c.weight, p.deposit_mode, normalize_npart);
    if (p.denoise) launch_denoise(c, normalize_npart);
  }
  stage_mark(c, 2);
  launch_deposit_coarse(c, c.weight, p.deposit_mode);
  if (normalize_npart > 0) launch_deposit_coarse_finish(c, p.deposit_mode);
  stage_mark(c, 3);
}

void enqueue_phase_fields(Ctx& c, const vlb_step_params& p, int64_t normalize_npart) {
  if (normalize_npart > 0) {
    launch_deposit_coarse_finish(c, p.deposit_mode);
    launch_deposit_fine_normalize(c, c.weight, p.deposit_mode, normalize_npart);
    if (p.denoise) launch_denoise(c, normalize_npart);
  }
  launch_poisson(c);
  stage_mark(c, 4);
  if (p.energy) {
    // the Hartree energy, on the Hartree potential alone (src/simulation.jl:505-513)
    launch_coefficients(c, c.fine, c.fine.phi, c.fine.csol_hartree);
    launch_energy(c, c.fine.csol_hartree, c.coarse.csol_hartree, &c.dsc->energy[0]);
  }
  launch_mean_field_coefficients(c, c.fine, c.fine.phi, c.fine.csol, p.jellium_nions, p.jellium_radius);
  launch_mean_field_coefficients(c, c.coarse, c.coarse.phi, c.coarse.csol, p.jellium_nions, p.jellium_radius);
  stage_mark(c, 5);
  launch_forces(c);
  stage_mark(c, 6);
}

void enqueue_phase_advance(Ctx& c, const vlb_step_params& p) {
  launch_projectile_update(c, p.dt, p.jellium_nions, p.jellium_radius, p.advance_projectile);
  stage_mark(c, 7);
  if (p.push) launch_push(c, p.dt, p.rcmax, p.capture_radius, true);
  stage_mark(c, 8);
  if (!p.push && p.capture_radius > 0) launch_enclosed(c, p.capture_radius);
  // the interaction with the total potential at the advanced positions
  // (src/simulation.jl:393-394)
  if (p.energy) launch_energy(c, c.fine.csol, c.coarse.csol, &c.dsc->energy[1]);
  // a film frame when the step asked for one (the kernels return at once
  // otherwise, so a captured step keeps them)
  if (c.film_cap > 0) launch_film(c, p.capture_radius);
  stage_mark(c, 9);
}

void enqueue_step(Ctx& c, const vlb_step_params& p) {
  enqueue_phase_deposit(c, p, c.N);
  enqueue_phase_fields(c, p, 0);
  enqueue_phase_advance(c, p);
}

bool same_params(const vlb_step_params& a, const vlb_step_params& b) {
  return a.dt == b.dt && a.rcmax == b.rcmax && a.jellium_nions == b.jellium_nions &&
         a.jellium_radius == b.jellium_radius && a.capture_radius == b.capture_radius &&
         a.deposit_mode == b.deposit_mode && a.advance_projectile == b.advance_projectile && a.push == b.push &&
         a.poisson_precision == b.poisson_precision && a.denoise == b.denoise && a.energy == b.energy;
}

// Two graphs, one per parity of the sort's double buffer: the step moves
// the cloud from part[cur] to part[cur^1], so graph g starts from cur == g.
void capture_graphs(Ctx& c, const vlb_step_params& p) {
  const int saved = c.cur;
  // the step's result reports the sort that ran eagerly, not the captured one
  const bool ran_near = c.last_sort_near;
  const long long launches0 = c.launches;
  for (int g = 0; g < 2; ++g) {
    if (c.gexec[g]) {
      VLB_CUDA(cudaGraphExecDestroy(c.gexec[g]));
      c.gexec[g] = nullptr;
    }
    c.cur = g;
    cudaGraph_t graph = nullptr;
    const long long l0 = c.launches;
    VLB_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_step(c, p);
    } catch (...) {
      cudaStreamEndCapture(c.stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      c.cur = saved;
      c.last_sort_near = ran_near;
      sync_sort_products(c);
      throw;
    }
    VLB_CUDA(cudaStreamEndCapture(c.stream, &graph));
    VLB_CUDA(cudaGraphInstantiate(&c.gexec[g], graph, 0));
    VLB_CUDA(cudaGraphDestroy(graph));
    if (g == 0) c.graph_launches = c.launches - l0;
  }
  c.launches = launches0;
  c.cur = saved;
  c.graph_sort_near = c.last_sort_near;
  c.last_sort_near = ran_near;
  sync_sort_products(c);
  c.graph_params = p;
  c.graph_valid = true;
}

}  // namespace

void set_last_error(const std::string& msg) { g_err = msg; }

std::string cuda_msg(cudaError_t e, const char* what) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

}  // namespace vlb

using namespace vlb;

extern "C" {

const char* vlb_last_error(void) { return g_err.c_str(); }
const char* vlb_version(void) { return "vlasov_b200 0.1 (sm_100a)"; }

int vlb_create(const vlb_config* cfg, vlb_ctx** out) {
  if (!cfg || !out) return fail(VLB_ERR_ARG, "null config or output handle");
  *out = nullptr;
  Ctx* c = nullptr;
  int rc = guarded([&]() -> int {
    if (cfg->npart < 1) throw ArgError("npart must be positive");
    if (cfg->npart > (int64_t)INT32_MAX / 2) throw ArgError("npart too large for 32-bit slots");
    if (!(cfg->weight > 0)) throw ArgError("weight must be positive");
    check_level(cfg->fine, "fine");
    check_level(cfg->coarse, "coarse");
    const vlb_smoothing_desc& S = cfg->smoothing;
    if (S.nbdt < 1 || !S.overlap || !S.gradient || !S.nodes) throw ArgError("smoothing tables missing");
    // the accelerated path assumes a uniform fine axis (src/accelerator.jl:262-268)
    const double* kf = cfg->fine.knots;
    const int nkf = cfg->fine.nknots;
    const double h = (kf[nkf - 1] - kf[0]) / (nkf - 1);
    for (int i = 1; i < nkf; ++i)
      if (std::fabs((kf[i] - kf[i - 1]) - h) > 1e-9 * std::fabs(h))
        throw ArgError("the accelerated path assumes a uniform fine grid");
    if (cfg->coarse.knots[0] > kf[0] || cfg->coarse.knots[cfg->coarse.nknots - 1] < kf[nkf - 1])
      throw ArgError("the fine level sticks out of the coarse level");
    int ndev = 0;
    VLB_CUDA(cudaGetDeviceCount(&ndev));
    if (cfg->device < 0 || cfg->device >= ndev) throw ArgError("no such CUDA device");
    c = new Ctx();
    c->device = cfg->device;
    VLB_CUDA(cudaSetDevice(c->device));
    VLB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
    VLB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->N = cfg->npart;
    c->Npad = (c->N + 63) / 64 * 64;
    c->weight = cfg->weight;
    setup_level(c->fine, cfg->fine, false);
    setup_level(c->coarse, cfg->coarse, true);
    c->x0 = kf[0];
    c->h = h;
    c->x0f = (float)c->x0;
    c->hf = (float)c->h;
    c->spacing_f = (float)S.spacing;
    const double half = S.spacing / 2;
    c->lo_f = (float)(kf[1] + half);
    c->hi_f = (float)(kf[nkf - 2] - half);
    c->nbdt = S.nbdt;
    c->ncol = S.nbdt + 1;
    c->overlap = upload_f(S.overlap, (size_t)c->ncol * 10);
    c->gradient = upload_f(S.gradient, (size_t)c->ncol * 10);
    {
      const std::vector<float> ov = to_float(S.overlap, (size_t)c->ncol * 10);
      const std::vector<float> gr = to_float(S.gradient, (size_t)c->ncol * 10);
      std::vector<float> both((size_t)c->ncol * 20);
      for (size_t col = 0; col < (size_t)c->ncol; ++col)
        for (int e = 0; e < 10; ++e) {
          both[col * 20 + e] = ov[col * 10 + e];
          both[col * 20 + 10 + e] = gr[col * 10 + e];
        }
      c->ovgr = upload(both.data(), both.size());
    }
    c->nodes = upload_f(S.nodes, (size_t)c->ncol * 8);
    const size_t P = 3 * (size_t)c->Npad;
    for (int b = 0; b < 2; ++b) {
      c->part[b].k = dalloc<int32_t>(P);
      c->part[b].d = dalloc<float>(P);
      c->part[b].pk = dalloc<int32_t>(P);
      c->part[b].pd = dalloc<float>(P);
      VLB_CUDA(cudaMemset(c->part[b].k, 0, P * 4));
      VLB_CUDA(cudaMemset(c->part[b].d, 0, P * 4));
      VLB_CUDA(cudaMemset(c->part[b].pk, 0, P * 4));
      VLB_CUDA(cudaMemset(c->part[b].pd, 0, P * 4));
    }
    c->force = dalloc<float>(P);
    VLB_CUDA(cudaMemset(c->force, 0, P * 4));
    const int64_t N = c->N;
    c->ncell = c->fine.nk * c->fine.nk * c->fine.nk;
    c->keys = dalloc<uint32_t>(N);
    c->keys_alt = dalloc<uint32_t>(N);
    c->skeys = dalloc<uint32_t>(N);
    c->perm = dalloc<uint32_t>(N);
    c->cols = dalloc<uint32_t>(N);
    c->cols_packed = c->ncol <= 1024;
    c->vals_alt = dalloc<uint32_t>(N);
    const int64_t ntiles = (N + 4095) / 4096;
    c->radix_table_size = 1024 * ntiles;
    c->radix_table = dalloc<uint32_t>(c->radix_table_size);
    c->counts = dalloc<int32_t>(c->ncell);
    c->cell_off = dalloc<int32_t>(c->ncell);
    for (int p = 0; p < 2; ++p) {
      c->occ_buf[p] = dalloc<int32_t>(c->ncell);
      c->bnd_buf[p] = dalloc<int32_t>(c->ncell + 1);
      c->cidx_buf[p] = dalloc<int32_t>(c->ncell);
      VLB_CUDA(cudaMemset(c->occ_buf[p], 0, (size_t)c->ncell * 4));
      VLB_CUDA(cudaMemset(c->bnd_buf[p], 0, ((size_t)c->ncell + 1) * 4));
      VLB_CUDA(cudaMemset(c->cidx_buf[p], 0, (size_t)c->ncell * 4));
    }
    c->occupied = c->occ_buf[0];
    c->bounds = c->bnd_buf[0];
    const size_t maxocc = (size_t)std::min<int64_t>(c->ncell, N);
    c->dir_cnt = dalloc<int32_t>(maxocc * 27);
    c->dir_base = dalloc<int32_t>(maxocc * 27);
    c->outlist = dalloc<int32_t>(N);
    for (int p = 0; p < 2; ++p) {
      c->cstart_buf[p] = dalloc<int32_t>(c->ncell);
      c->item_buf[p] = dalloc<int32_t>(N / kMinChunk + c->ncell + 1);
      c->rec_buf[p] = dalloc<int4>((size_t)N / kMinChunk + c->ncell + 1);
    }
    c->chunk_start = c->cstart_buf[0];
    c->item_cell = c->item_buf[0];
    c->item_dir = dalloc<int32_t>(((size_t)N / kMinChunk + c->ncell + 1) * 27);
    c->item_rec = c->rec_buf[0];
    const int64_t scan_tiles = std::max<int64_t>({(N + 4095) / 4096, (c->ncell + 4095) / 4096,
                                                  (c->radix_table_size + 4095) / 4096}) + 1;
    c->scan_status_size = 8 * scan_tiles;
    c->scan_status = dalloc<unsigned long long>(c->scan_status_size);
    const int nf = c->fine.n, nc = c->coarse.n;
    const size_t maxg = (size_t)std::max(nf, nc) * std::max(nf, nc) * std::max(nf, nc);
    c->rho_fixed = dalloc<unsigned long long>((size_t)nf * nf * nf);
    c->rho_fixed_c = dalloc<unsigned long long>((size_t)nc * nc * nc);
    c->red_items = dalloc<double>(4 * (size_t)(N / kMinChunk + c->ncell + 1));
    c->red_tail = dalloc<double>(4 * (size_t)c->num_sms);
    c->red_blocks = dalloc<double>(4 * (size_t)c->num_sms);
    c->e_items = dalloc<double>((size_t)(N / kMinChunk + c->ncell + 1));
    c->e_blocks = dalloc<double>((size_t)c->num_sms);
    c->diag_part = dalloc<double>(5 * (size_t)c->num_sms * 32);
    c->partials = dalloc<double>(10 * (size_t)std::max(nf, nc) * std::max(nf, nc));
    for (auto& w : c->work) w = dalloc<float>(maxg);
    c->dsc = dalloc<DeviceScalars>(1);
    VLB_CUDA(cudaMemset(c->dsc, 0, sizeof(DeviceScalars)));
    VLB_CUDA(cudaMallocHost(&c->hsc, sizeof(DeviceScalars)));
    VLB_CUDA(cudaMallocHost(&c->hin, sizeof(DeviceScalars)));
    memset(c->hsc, 0, sizeof(DeviceScalars));
    memset(c->hin, 0, sizeof(DeviceScalars));
    for (auto& e : c->ev) VLB_CUDA(cudaEventCreate(&e));
    c->evs_made = true;
    deposit_setup(*c);
    field_setup(*c);
    tc_setup(*c);
    VLB_CUDA(cudaDeviceSynchronize());
    return VLB_OK;
  });
  if (rc != VLB_OK) {
    std::string msg = g_err;
    destroy_ctx(c);
    g_err = msg;
    return rc;
  }
  *out = reinterpret_cast<vlb_ctx*>(c);
  return VLB_OK;
}

int vlb_destroy(vlb_ctx* ctx) {
  if (!ctx) return fail(VLB_ERR_ARG, "null context");
  destroy_ctx(reinterpret_cast<Ctx*>(ctx));
  return VLB_OK;
}

#define CTX_OR_FAIL                                              \
  if (!ctx) return fail(VLB_ERR_ARG, "null context");            \
  Ctx& c = *reinterpret_cast<Ctx*>(ctx);                         \
  if (cudaSetDevice(c.device) != cudaSuccess) return fail(VLB_ERR_CUDA, "cudaSetDevice failed")

int vlb_upload_particles(vlb_ctx* ctx, const int32_t* knode, const float* delta, const int32_t* pknode,
                         const float* pdelta) {
  CTX_OR_FAIL;
  if (!knode || !delta || !pknode || !pdelta) return fail(VLB_ERR_ARG, "null particle array");
  return guarded([&]() -> int {
    Particles& P = c.part[c.cur];
    const size_t n = (size_t)c.N;
    for (int a = 0; a < 3; ++a) {
      VLB_CUDA(cudaMemcpyAsync(P.k + a * c.Npad, knode + a * n, n * 4, cudaMemcpyHostToDevice, c.stream));
      VLB_CUDA(cudaMemcpyAsync(P.d + a * c.Npad, delta + a * n, n * 4, cudaMemcpyHostToDevice, c.stream));
      VLB_CUDA(cudaMemcpyAsync(P.pk + a * c.Npad, pknode + a * n, n * 4, cudaMemcpyHostToDevice, c.stream));
      VLB_CUDA(cudaMemcpyAsync(P.pd + a * c.Npad, pdelta + a * n, n * 4, cudaMemcpyHostToDevice, c.stream));
    }
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    c.prev_deferred = false;  // every slot's previous position was just written
    c.sorted = false;
    c.items_valid = false;
    c.keys_ready = false;
    c.order_valid = false;
    return VLB_OK;
  });
}

int vlb_download_particles(vlb_ctx* ctx, int32_t* knode, float* delta, int32_t* pknode, float* pdelta) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    if (pknode || pdelta) settle_prev(c);
    Particles& P = c.part[c.cur];
    const size_t n = (size_t)c.N;
    for (int a = 0; a < 3; ++a) {
      if (knode) VLB_CUDA(cudaMemcpyAsync(knode + a * n, P.k + a * c.Npad, n * 4, cudaMemcpyDeviceToHost, c.stream));
      if (delta) VLB_CUDA(cudaMemcpyAsync(delta + a * n, P.d + a * c.Npad, n * 4, cudaMemcpyDeviceToHost, c.stream));
      if (pknode) VLB_CUDA(cudaMemcpyAsync(pknode + a * n, P.pk + a * c.Npad, n * 4, cudaMemcpyDeviceToHost, c.stream));
      if (pdelta) VLB_CUDA(cudaMemcpyAsync(pdelta + a * n, P.pd + a * c.Npad, n * 4, cudaMemcpyDeviceToHost, c.stream));
    }
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

// Slots [first, first + count) of the cloud, from or to host SoA arrays of
// 3*count (all x, then all y, then all z): the chunked form of upload!/
// download!, so that a cloud can be built or read a slice at a time.
int vlb_upload_particles_range(vlb_ctx* ctx, int64_t first, int64_t count, const int32_t* knode, const float* delta,
                               const int32_t* pknode, const float* pdelta) {
  CTX_OR_FAIL;
  if (!knode || !delta || !pknode || !pdelta) return fail(VLB_ERR_ARG, "null particle array");
  if (first < 0 || count < 0 || first > c.N || count > c.N - first)
    return fail(VLB_ERR_ARG, "vlb_upload_particles_range: slots out of the cloud");
  return guarded([&]() -> int {
    settle_prev(c);  // the slots outside the range keep their previous positions
    Particles& P = c.part[c.cur];
    const size_t n = (size_t)count, bytes = n * 4;
    if (n) {
      for (int a = 0; a < 3; ++a) {
        const size_t o = a * (size_t)c.Npad + (size_t)first;
        VLB_CUDA(cudaMemcpyAsync(P.k + o, knode + a * n, bytes, cudaMemcpyHostToDevice, c.stream));
        VLB_CUDA(cudaMemcpyAsync(P.d + o, delta + a * n, bytes, cudaMemcpyHostToDevice, c.stream));
        VLB_CUDA(cudaMemcpyAsync(P.pk + o, pknode + a * n, bytes, cudaMemcpyHostToDevice, c.stream));
        VLB_CUDA(cudaMemcpyAsync(P.pd + o, pdelta + a * n, bytes, cudaMemcpyHostToDevice, c.stream));
      }
    }
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    c.sorted = false;
    c.items_valid = false;
    c.keys_ready = false;
    c.order_valid = false;
    return VLB_OK;
  });
}

int vlb_download_particles_range(vlb_ctx* ctx, int64_t first, int64_t count, int32_t* knode, float* delta,
                                 int32_t* pknode, float* pdelta) {
  CTX_OR_FAIL;
  if (first < 0 || count < 0 || first > c.N || count > c.N - first)
    return fail(VLB_ERR_ARG, "vlb_download_particles_range: slots out of the cloud");
  return guarded([&]() -> int {
    if (pknode || pdelta) settle_prev(c);
    Particles& P = c.part[c.cur];
    const size_t n = (size_t)count, bytes = n * 4;
    if (n) {
      for (int a = 0; a < 3; ++a) {
        const size_t o = a * (size_t)c.Npad + (size_t)first;
        if (knode) VLB_CUDA(cudaMemcpyAsync(knode + a * n, P.k + o, bytes, cudaMemcpyDeviceToHost, c.stream));
        if (delta) VLB_CUDA(cudaMemcpyAsync(delta + a * n, P.d + o, bytes, cudaMemcpyDeviceToHost, c.stream));
        if (pknode) VLB_CUDA(cudaMemcpyAsync(pknode + a * n, P.pk + o, bytes, cudaMemcpyDeviceToHost, c.stream));
        if (pdelta) VLB_CUDA(cudaMemcpyAsync(pdelta + a * n, P.pd + o, bytes, cudaMemcpyDeviceToHost, c.stream));
      }
    }
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_get_forces_range(vlb_ctx* ctx, int64_t first, int64_t count, float* host) {
  CTX_OR_FAIL;
  if (!host) return fail(VLB_ERR_ARG, "null host buffer");
  if (first < 0 || count < 0 || first > c.N || count > c.N - first)
    return fail(VLB_ERR_ARG, "vlb_get_forces_range: slots out of the cloud");
  return guarded([&]() -> int {
    const size_t n = (size_t)count;
    if (n)
      for (int a = 0; a < 3; ++a)
        VLB_CUDA(cudaMemcpyAsync(host + a * n, c.force + a * (size_t)c.Npad + (size_t)first, n * 4,
                                 cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_sort(vlb_ctx* ctx, int32_t* noccupied, int32_t* outcount) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    reset_step_scalars(c);
    launch_sort(c, false);
    fetch_scalars(c);
    if (noccupied) *noccupied = c.hsc->noccupied;
    if (outcount) *outcount = c.hsc->outcount;
    return status_code(c);
  });
}

int vlb_get_sort(vlb_ctx* ctx, int32_t* perm, int32_t* occupied, int32_t* bounds, int32_t* outlist) {
  CTX_OR_FAIL;
  if (!c.sorted) return fail(VLB_ERR_STATE, "no sort has run on the current cloud");
  return guarded([&]() -> int {
    fetch_scalars(c);
    const int nocc = c.hsc->noccupied, nout = c.hsc->outcount;
    if (perm) VLB_CUDA(cudaMemcpyAsync(perm, c.perm, (size_t)c.N * 4, cudaMemcpyDeviceToHost, c.stream));
    if (occupied) VLB_CUDA(cudaMemcpyAsync(occupied, c.occupied, (size_t)nocc * 4, cudaMemcpyDeviceToHost, c.stream));
    if (bounds) VLB_CUDA(cudaMemcpyAsync(bounds, c.bounds, (size_t)(nocc + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
    if (outlist && nout)
      VLB_CUDA(cudaMemcpyAsync(outlist, c.outlist, (size_t)nout * 4, cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_get_sort_sizes(vlb_ctx* ctx, int32_t* noccupied, int32_t* outcount) {
  CTX_OR_FAIL;
  if (!c.sorted) return fail(VLB_ERR_STATE, "no sort has run on the current cloud");
  return guarded([&]() -> int {
    fetch_scalars(c);
    if (noccupied) *noccupied = c.hsc->noccupied;
    if (outcount) *outcount = c.hsc->outcount;
    return VLB_OK;
  });
}

int vlb_deposit_fine(vlb_ctx* ctx, double charge, int32_t mode, int32_t* nout, double* total_charge) {
  CTX_OR_FAIL;
  if (mode != VLB_DEPOSIT_FLOAT32 && mode != VLB_DEPOSIT_FIXED64) return fail(VLB_ERR_ARG, "unknown deposit mode");
  if (!c.sorted) return fail(VLB_ERR_STATE, "deposit before any sort of the current cloud");
  return guarded([&]() -> int {
    launch_deposit_fine(c, charge, mode);
    fetch_scalars(c);
    if (nout) *nout = c.hsc->nout;
    if (total_charge) *total_charge = c.hsc->charge_raw;
    return status_code(c);
  });
}

int vlb_deposit_coarse(vlb_ctx* ctx, double charge) {
  CTX_OR_FAIL;
  if (!c.sorted) return fail(VLB_ERR_STATE, "deposit before any sort of the current cloud");
  return guarded([&]() -> int {
    launch_deposit_coarse(c, charge, VLB_DEPOSIT_FLOAT32);
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

namespace {
int check_precision(const Ctx& c, int32_t precision) {
  if (precision == VLB_POISSON_FP32) return VLB_OK;
  if (precision != VLB_POISSON_3XTF32 && precision != VLB_POISSON_BF16X3)
    return fail(VLB_ERR_ARG, "unknown mode-product precision");
  if (!c.fine.tc_sinv.img || !c.fine.tc_M.img || !c.coarse.tc_sinv.img || !c.coarse.tc_M.img)
    return fail(VLB_ERR_ARG, "tensor-core mode products need an even n <= 144 points per axis on both levels");
  return VLB_OK;
}
}  // namespace

int vlb_set_precision(vlb_ctx* ctx, int32_t precision) {
  CTX_OR_FAIL;
  if (int rc = check_precision(c, precision)) return rc;
  c.mode_precision = precision;
  return VLB_OK;
}

int vlb_poisson(vlb_ctx* ctx, int32_t precision) {
  CTX_OR_FAIL;
  if (int rc = check_precision(c, precision)) return rc;
  c.mode_precision = precision;
  return guarded([&]() -> int {
    VLB_CUDA(cudaMemsetAsync(&c.dsc->status, 0, sizeof(int32_t), c.stream));
    launch_poisson(c);
    fetch_scalars(c);
    return status_code(c);
  });
}

int vlb_coefficients(vlb_ctx* ctx, int32_t level) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    Level& L = level_of(c, level);
    VLB_CUDA(cudaMemsetAsync(&c.dsc->status, 0, sizeof(int32_t), c.stream));
    launch_coefficients(c, L, L.phi, L.csol);
    fetch_scalars(c);
    return status_code(c);
  });
}

int vlb_mean_field(vlb_ctx* ctx, int32_t level, double nions, double radius) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    Level& L = level_of(c, level);
    VLB_CUDA(cudaMemsetAsync(&c.dsc->status, 0, sizeof(int32_t), c.stream));
    launch_mean_field_add(c, L, nions, radius);
    fetch_scalars(c);
    return status_code(c);
  });
}

int vlb_forces(vlb_ctx* ctx, const vlb_projectile* proj, double red[4], int32_t* outcount) {
  CTX_OR_FAIL;
  if (!c.sorted) return fail(VLB_ERR_STATE, "forces before any sort of the current cloud");
  return guarded([&]() -> int {
    upload_projectile(c, proj);
    launch_forces(c);
    fetch_scalars(c);
    if (red)
      for (int i = 0; i < 4; ++i) red[i] = c.hsc->red[i];
    if (outcount) *outcount = c.hsc->outcount;
    return status_code(c);
  });
}

int vlb_projectile_forces(vlb_ctx* ctx, const vlb_projectile* proj, double nions, double jellium_radius,
                          double force[3], double* e_electrons, double* e_jellium) {
  CTX_OR_FAIL;
  if (!proj) return fail(VLB_ERR_ARG, "null projectile");
  if (!c.have_forces) return fail(VLB_ERR_STATE, "projectile forces before any force evaluation");
  // host scalar arithmetic on the sums of the last vlb_forces (src/accelerator.jl:746-756)
  const double* P = proj->position;
  const double q = proj->charge;
  const double r2 = P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
  const double modf = r2 > jellium_radius * jellium_radius ? nions * q / std::pow(r2, 1.5) : q / 64.0;
  for (int d = 0; d < 3; ++d)
    if (force) force[d] = modf * P[d] + c.hsc->red[d];
  if (e_electrons) *e_electrons = c.weight * q * c.hsc->red[3];
  const double r = std::sqrt(r2);
  if (e_jellium)
    *e_jellium = q * (r < jellium_radius ? -nions * (3 - (r / jellium_radius) * (r / jellium_radius)) / (2 * jellium_radius)
                                         : -nions / r);
  return VLB_OK;
}

int vlb_push(vlb_ctx* ctx, double dt, double rcmax, double diag[5]) {
  CTX_OR_FAIL;
  if (!(dt > 0)) return fail(VLB_ERR_ARG, "dt must be positive");
  return guarded([&]() -> int {
    launch_push(c, dt, rcmax, 0.0, false);
    fetch_scalars(c);
    if (diag)
      for (int i = 0; i < 5; ++i) diag[i] = c.hsc->diag[i];
    c.sorted = false;  // the cloud moved: the cell lists are stale
    return VLB_OK;
  });
}

namespace {
int check_step_params(Ctx& c, const vlb_step_params* params) {
  if (!params) return fail(VLB_ERR_ARG, "null step parameters");
  if (!(params->dt > 0)) return fail(VLB_ERR_ARG, "dt must be positive");
  if (params->deposit_mode != VLB_DEPOSIT_FLOAT32 && params->deposit_mode != VLB_DEPOSIT_FIXED64)
    return fail(VLB_ERR_ARG, "unknown deposit mode");
  if (params->denoise && !c.dn) return fail(VLB_ERR_STATE, "denoise asked for, and no denoiser is set");
  if (params->film && c.film_cap <= 0) return fail(VLB_ERR_STATE, "a film frame asked for, and no film is reserved");
  return check_precision(c, params->poisson_precision);
}

// Scalars back to the host after a step (synchronises the stream), the
// projectile out, the step's results.
void collect_step(Ctx& c, vlb_projectile* proj, const vlb_step_params* params, vlb_step_result* result);

void finish_step(Ctx& c, vlb_projectile* proj, const vlb_step_params* params, vlb_step_result* result) {
  VLB_CUDA(cudaMemcpyAsync(c.hsc, c.dsc, sizeof(DeviceScalars), cudaMemcpyDeviceToHost, c.stream));
  VLB_CUDA(cudaStreamSynchronize(c.stream));
  collect_step(c, proj, params, result);
}

// The host side of a finished step, from the scalars already in c.hsc.
void collect_step(Ctx& c, vlb_projectile* proj, const vlb_step_params* params, vlb_step_result* result) {
  if (c.profile) {
    for (int i = 0; i < 9; ++i) {
      float ms = 0;
      VLB_CUDA(cudaEventElapsedTime(&ms, c.ev[i], c.ev[i + 1]));
      c.stage_ms[i] += ms;
    }
    // the gather kernel alone (its pair of events is recorded by launch_forces)
    float ms = 0;
    VLB_CUDA(cudaEventElapsedTime(&ms, c.ev[kEvGatherBegin], c.ev[kEvGatherEnd]));
    c.stage_ms[kEvGatherBegin] += ms;
  }
  c.sorted = false;  // after the push the lists describe the previous positions
  c.have_forces = true;
  const DeviceScalars& h = *c.hsc;
  if (proj) {
    for (int d = 0; d < 3; ++d) {
      proj->position[d] = h.proj_pos[d];
      proj->previous[d] = h.proj_prev[d];
      proj->velocity[d] = h.proj_vel[d];
    }
  }
  if (result) {
    result->kinetic = h.diag[0];
    result->escaped = h.diag[1];
    for (int d = 0; d < 3; ++d) {
      result->angular[d] = h.diag[2 + d];
      result->projectile_force[d] = h.proj_force[d];
    }
    result->e_electrons = h.e_el;
    result->e_jellium = h.e_jel;
    result->enclosed_charge = c.weight * (double)h.enclosed;
    result->total_charge = h.charge_raw;
    result->nout = h.nout;
    result->outcount = h.outcount;
    result->noccupied = h.noccupied;
    result->status = h.status;
    result->denoised = h.denoised;
    result->sort_path = c.last_sort_near ? (h.sort_far ? 2 : 1) : 0;
    result->hartree = params->energy ? 0.5 * h.energy[0] : 0.0;
    result->interaction = params->energy ? h.energy[1] : 0.0;
  }
  if (!params->push) c.sorted = true;  // forces-only: the cloud did not move
}
}  // namespace

int vlb_step(vlb_ctx* ctx, vlb_projectile* proj, const vlb_step_params* params, vlb_step_result* result) {
  CTX_OR_FAIL;
  if (int rc = check_step_params(c, params)) return rc;
  c.mode_precision = params->poisson_precision;
  return guarded([&]() -> int {
    c.shard_phase = 0;
    upload_projectile(c, proj, params->film ? 1 : 0);
    const bool graph = params->use_graph && !c.profile;
    // the captured step starts from keys written by the previous push
    if (graph && c.graph_valid && c.keys_ready && same_params(c.graph_params, *params)) {
      const int g = c.cur;
      VLB_CUDA(cudaGraphLaunch(c.gexec[g], c.stream));
      c.launches += c.graph_launches;
      c.cur ^= 1;
      c.last_sort_near = c.graph_sort_near;
      sync_sort_products(c);
    } else {
      const long long before = c.launches;
      enqueue_step(c, *params);
      c.graph_launches = c.launches - before;
      if (graph) {
        // the eager run above did this step's work; capture for the next ones
        const long long keep = c.launches;
        capture_graphs(c, *params);
        c.launches = keep;
      }
    }
    finish_step(c, proj, params, result);
    return status_code(c);
  });
}

// ----------------------------------------------------------- denoiser
int vlb_set_denoiser(vlb_ctx* ctx, const float* weights, int32_t count, double input_scale,
                     double charge_tolerance) {
  CTX_OR_FAIL;
  if (!weights || count != vlb_dn_weight_count())
    return fail(VLB_ERR_ARG, "vlb_set_denoiser: expected " + std::to_string(vlb_dn_weight_count()) + " weights");
  if (!(input_scale > 0) || !(charge_tolerance >= 0)) return fail(VLB_ERR_ARG, "vlb_set_denoiser: bad scale or tolerance");
  return guarded([&]() -> int {
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    free_denoiser(c);
    ++c.config_epoch;
    const int n = c.fine.n;
    c.dn = dn_create(n, n, n, c.device, c.num_sms);
    dn_route_status(c.dn, &c.dsc->status);  // a timed-out wait shows in the step's status
    std::vector<float> w(weights, weights + count);
    for (float& f : w) {  // round to BF16, ties to even
      uint32_t u;
      std::memcpy(&u, &f, 4);
      u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
      std::memcpy(&f, &u, 4);
    }
    c.dn_weights = dalloc<float>(w.size());
    VLB_CUDA(cudaMemcpy(c.dn_weights, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
    c.dn_pred = dalloc<float>((size_t)n * n * n);
    c.dn_scale = input_scale;
    c.dn_tol = charge_tolerance;
    c.graph_valid = false;
    return VLB_OK;
  });
}

int vlb_clear_denoiser(vlb_ctx* ctx) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    free_denoiser(c);
    ++c.config_epoch;
    c.graph_valid = false;
    return VLB_OK;
  });
}

// ------------------------------------------------------------ film
int vlb_film_reserve(vlb_ctx* ctx, int32_t capacity, int32_t iz1, int32_t iz2, double radius) {
  CTX_OR_FAIL;
  const int n = c.fine.n;
  if (capacity < 1 || iz1 < 0 || iz1 >= n || iz2 < 0 || iz2 >= n || !(radius >= 0))
    return fail(VLB_ERR_ARG, "vlb_film_reserve: capacity >= 1, planes in [0, n) and radius >= 0 are required");
  if ((size_t)capacity * n * n > ((size_t)1 << 34))
    return fail(VLB_ERR_ARG, "vlb_film_reserve: more than 64 GB of frames");
  return guarded([&]() -> int {
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    dfree(c.film_frames);
    dfree(c.film_scalars);
    c.film_cap = 0;
    c.film_frames = dalloc<float>((size_t)capacity * n * n);
    c.film_scalars = dalloc<double>(4 * (size_t)capacity);
    VLB_CUDA(cudaMemset(&c.dsc->film_next, 0, sizeof(int32_t)));
    VLB_CUDA(cudaMemset(&c.dsc->film_inside, 0, sizeof(unsigned long long)));
    c.film_cap = capacity;
    c.film_iz1 = iz1;
    c.film_iz2 = iz2;
    c.film_r2 = radius * radius;
    c.graph_valid = false;  // the captured step gains the film's kernels
    ++c.config_epoch;
    return VLB_OK;
  });
}

int vlb_film_frames(vlb_ctx* ctx, int32_t* taken, int32_t* stored) {
  CTX_OR_FAIL;
  if (c.film_cap <= 0) return fail(VLB_ERR_STATE, "vlb_film_frames: no film is reserved");
  return guarded([&]() -> int {
    int32_t next = 0;
    VLB_CUDA(cudaMemcpyAsync(&next, &c.dsc->film_next, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    if (taken) *taken = next;
    if (stored) *stored = next < c.film_cap ? next : c.film_cap;
    return VLB_OK;
  });
}

int vlb_film_download(vlb_ctx* ctx, int32_t first, int32_t count, float* frames, double* scalars) {
  CTX_OR_FAIL;
  if (c.film_cap <= 0) return fail(VLB_ERR_STATE, "vlb_film_download: no film is reserved");
  if (first < 0 || count < 0 || (int64_t)first + (int64_t)count > (int64_t)c.film_cap)
    return fail(VLB_ERR_ARG, "vlb_film_download: frames out of the reserved range");
  const size_t nn = (size_t)c.fine.n * c.fine.n;
  return guarded([&]() -> int {
    if (frames && count)
      VLB_CUDA(cudaMemcpyAsync(frames, c.film_frames + (size_t)first * nn, (size_t)count * nn * sizeof(float),
                               cudaMemcpyDeviceToHost, c.stream));
    if (scalars && count)
      VLB_CUDA(cudaMemcpyAsync(scalars, c.film_scalars + 4 * (size_t)first, 4 * (size_t)count * sizeof(double),
                               cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_film_clear(vlb_ctx* ctx) {
  CTX_OR_FAIL;
  return guarded([&]() -> int {
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    dfree(c.film_frames);
    dfree(c.film_scalars);
    c.film_frames = nullptr;
    c.film_scalars = nullptr;
    c.film_cap = 0;
    c.graph_valid = false;
    ++c.config_epoch;
    return VLB_OK;
  });
}

// ------------------------------------------------------------ energy
int vlb_interaction_energy(vlb_ctx* ctx, int32_t coefficients, double* out) {
  CTX_OR_FAIL;
  if (!out || (coefficients != VLB_ENERGY_TOTAL && coefficients != VLB_ENERGY_HARTREE))
    return fail(VLB_ERR_ARG, "vlb_interaction_energy: bad arguments");
  if (!c.items_valid) return fail(VLB_ERR_STATE, "interaction energy before any sort of the cloud");
  return guarded([&]() -> int {
    const int which = coefficients == VLB_ENERGY_HARTREE ? 0 : 1;
    launch_energy(c, which ? c.fine.csol : c.fine.csol_hartree, which ? c.coarse.csol : c.coarse.csol_hartree,
                  &c.dsc->energy[which]);
    fetch_scalars(c);
    *out = c.hsc->energy[which];
    return status_code(c);
  });
}

// ------------------------------------------------------------ tuning
int vlb_set_tuning(vlb_ctx* ctx, const vlb_tuning* t) {
  CTX_OR_FAIL;
  if (!t) return fail(VLB_ERR_ARG, "null tuning");
  if (t->chunk < kMinChunk || t->chunk > 4096 || t->chunk % 32)
    return fail(VLB_ERR_ARG, "chunk must be a multiple of 32 in [32, 4096]");
  const int32_t cps[4] = {t->field_ctas_per_sm, t->cic_ctas_per_sm, t->push_ctas_per_sm, t->move_ctas_per_sm};
  for (int32_t v : cps)
    if (v < 1 || v > 32) return fail(VLB_ERR_ARG, "CTAs per SM must be in [1, 32]");
  if (t->field_tensor_cores != 0 && t->field_tensor_cores != 1)
    return fail(VLB_ERR_ARG, "field_tensor_cores must be 0 or 1");
  if (t->scan_wait_polls < -1) return fail(VLB_ERR_ARG, "scan_wait_polls must be -1, 0 or positive");
  c.chunk = t->chunk;
  c.field_tc = t->field_tensor_cores != 0;
  c.field_cps = t->field_ctas_per_sm;
  c.cic_cps = t->cic_ctas_per_sm;
  c.push_cps = t->push_ctas_per_sm;
  c.move_cps = t->move_ctas_per_sm;
  c.scan_wait_polls = t->scan_wait_polls;
  c.graph_valid = false;  // the captured step has the old launch shapes
  ++c.config_epoch;
  c.sorted = false;       // the work items follow the chunk
  c.items_valid = false;
  return VLB_OK;
}

int vlb_get_tuning(vlb_ctx* ctx, vlb_tuning* t) {
  CTX_OR_FAIL;
  if (!t) return fail(VLB_ERR_ARG, "null tuning");
  *t = vlb_tuning{};
  t->chunk = c.chunk;
  t->field_ctas_per_sm = c.field_cps;
  t->cic_ctas_per_sm = c.cic_cps;
  t->push_ctas_per_sm = c.push_cps;
  t->move_ctas_per_sm = c.move_cps;
  t->field_tensor_cores = c.field_tc ? 1 : 0;
  t->scan_wait_polls = c.scan_wait_polls;
  return VLB_OK;
}

// ------------------------------------------------------------- batches
struct vlb_batch {
  std::vector<Ctx*> ctx;
  int device = 0;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  std::vector<int> cur0;       // the contexts' sort parities that gexec[0] starts from
  std::vector<uint64_t> epoch0;  // the contexts' configuration epochs the graphs were captured at
  vlb_step_params params{};
  bool valid = false;
};

namespace {

// One step of every context of the batch, each on its own stream, forked
// from and joined back to the batch's stream.
void enqueue_batch(vlb_batch& b, const vlb_step_params& p) {
  VLB_CUDA(cudaEventRecord(b.fork, b.origin));
  for (size_t i = 0; i < b.ctx.size(); ++i) {
    Ctx& c = *b.ctx[i];
    VLB_CUDA(cudaStreamWaitEvent(c.stream, b.fork, 0));
    enqueue_step(c, p);
    VLB_CUDA(cudaEventRecord(b.join[i], c.stream));
    VLB_CUDA(cudaStreamWaitEvent(b.origin, b.join[i], 0));
  }
}

void destroy_batch_graphs(vlb_batch& b) {
  for (auto& g : b.gexec) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  b.valid = false;
}

// Two graphs: from the contexts' current parities, and from all flipped.
void capture_batch(vlb_batch& b, const vlb_step_params& p) {
  destroy_batch_graphs(b);
  std::vector<int> saved(b.ctx.size());
  std::vector<char> ran_near(b.ctx.size());  // the results report the sorts that ran eagerly
  for (size_t i = 0; i < b.ctx.size(); ++i) {
    saved[i] = b.ctx[i]->cur;
    ran_near[i] = b.ctx[i]->last_sort_near;
  }
  b.cur0 = saved;
  for (int g = 0; g < 2; ++g) {
    for (size_t i = 0; i < b.ctx.size(); ++i) {
      b.ctx[i]->cur = saved[i] ^ g;
      b.ctx[i]->keys_ready = true;  // the captured step follows a step whose push wrote them
    }
    cudaGraph_t graph = nullptr;
    std::vector<long long> l0(b.ctx.size());
    for (size_t i = 0; i < b.ctx.size(); ++i) l0[i] = b.ctx[i]->launches;
    VLB_CUDA(cudaStreamBeginCapture(b.origin, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_batch(b, p);
    } catch (...) {
      cudaStreamEndCapture(b.origin, &graph);
      if (graph) cudaGraphDestroy(graph);
      for (size_t i = 0; i < b.ctx.size(); ++i) {
        b.ctx[i]->cur = saved[i];
        b.ctx[i]->last_sort_near = ran_near[i];
        sync_sort_products(*b.ctx[i]);
      }
      throw;
    }
    VLB_CUDA(cudaStreamEndCapture(b.origin, &graph));
    cudaError_t e = cudaGraphInstantiate(&b.gexec[g], graph, 0);
    cudaGraphDestroy(graph);
    VLB_CUDA(e);
    if (g == 0)
      for (size_t i = 0; i < b.ctx.size(); ++i) b.ctx[i]->graph_launches = b.ctx[i]->launches - l0[i];
  }
  for (size_t i = 0; i < b.ctx.size(); ++i) {
    b.ctx[i]->cur = saved[i];
    b.ctx[i]->graph_sort_near = b.ctx[i]->last_sort_near;
    b.ctx[i]->last_sort_near = ran_near[i];
    sync_sort_products(*b.ctx[i]);
    b.ctx[i]->keys_ready = true;
  }
  b.epoch0.resize(b.ctx.size());
  for (size_t i = 0; i < b.ctx.size(); ++i) b.epoch0[i] = b.ctx[i]->config_epoch;
  b.params = p;
  b.valid = true;
}

}  // namespace

int vlb_batch_create(vlb_ctx* const* ctxs, int32_t n, vlb_batch** out) {
  if (!ctxs || !out || n < 1) return fail(VLB_ERR_ARG, "a batch needs at least one context");
  *out = nullptr;
  auto* b = new (std::nothrow) vlb_batch();
  if (!b) return fail(VLB_ERR_NOMEM, "batch");
  for (int32_t i = 0; i < n; ++i) {
    if (!ctxs[i]) {
      delete b;
      return fail(VLB_ERR_ARG, "null context in the batch");
    }
    Ctx* c = reinterpret_cast<Ctx*>(ctxs[i]);
    for (Ctx* o : b->ctx)
      if (o == c) {
        delete b;
        return fail(VLB_ERR_ARG, "a context appears twice in the batch");
      }
    if (i > 0 && c->device != b->ctx[0]->device) {
      delete b;
      return fail(VLB_ERR_ARG, "the contexts of a batch must share one device");
    }
    b->ctx.push_back(c);
  }
  b->device = b->ctx[0]->device;
  int rc = guarded([&]() -> int {
    VLB_CUDA(cudaSetDevice(b->device));
    VLB_CUDA(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking));
    VLB_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    b->join.assign(b->ctx.size(), nullptr);
    for (auto& e : b->join) VLB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return VLB_OK;
  });
  if (rc != VLB_OK) {
    vlb_batch_destroy(b);
    return rc;
  }
  *out = b;
  return VLB_OK;
}

int vlb_batch_destroy(vlb_batch* b) {
  if (!b) return VLB_OK;
  cudaSetDevice(b->device);
  if (b->origin) cudaStreamSynchronize(b->origin);
  destroy_batch_graphs(*b);
  for (auto& e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
  return VLB_OK;
}

int vlb_batch_step(vlb_batch* b, vlb_projectile* projs, const vlb_step_params* params, vlb_step_result* results) {
  if (!b) return fail(VLB_ERR_ARG, "null batch");
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(VLB_ERR_CUDA, "cudaSetDevice failed");
  for (Ctx* c : b->ctx) {
    if (int rc = check_step_params(*c, params)) return rc;
    if (c->profile) return fail(VLB_ERR_STATE, "a batch step cannot be profiled");
  }
  if (!params->push) return fail(VLB_ERR_ARG, "a batch step pushes the clouds");
  if (params->film) return fail(VLB_ERR_ARG, "a batch step takes no film frames (params.film must be 0)");
  return guarded([&]() -> int {
    const size_t n = b->ctx.size();
    for (size_t i = 0; i < n; ++i) {
      Ctx& c = *b->ctx[i];
      c.mode_precision = params->poisson_precision;
      c.shard_phase = 0;
      upload_projectile(c, projs ? &projs[i] : nullptr);
      VLB_CUDA(cudaEventRecord(b->join[i], c.stream));
      VLB_CUDA(cudaStreamWaitEvent(b->origin, b->join[i], 0));
    }
    // the captured steps start from keys written by the previous pushes and
    // from the parities they were captured at
    bool replay = params->use_graph && b->valid && same_params(b->params, *params);
    int g = -1;
    if (replay) {
      bool same = true, flipped = true;
      for (size_t i = 0; i < n; ++i) {
        const Ctx& c = *b->ctx[i];
        replay = replay && c.keys_ready && c.config_epoch == b->epoch0[i];
        same = same && c.cur == b->cur0[i];
        flipped = flipped && c.cur == (b->cur0[i] ^ 1);
      }
      g = same ? 0 : (flipped ? 1 : -1);
      replay = replay && g >= 0;
    }
    if (replay) {
      VLB_CUDA(cudaGraphLaunch(b->gexec[g], b->origin));
      for (Ctx* c : b->ctx) {
        c->cur ^= 1;
        c->last_sort_near = c->graph_sort_near;
        sync_sort_products(*c);
        c->keys_ready = true;
        c->launches += c->graph_launches;
      }
    } else {
      std::vector<long long> before(n);
      for (size_t i = 0; i < n; ++i) before[i] = b->ctx[i]->launches;
      enqueue_batch(*b, *params);
      for (size_t i = 0; i < n; ++i) b->ctx[i]->graph_launches = b->ctx[i]->launches - before[i];
      if (params->use_graph) {
        std::vector<long long> keep(n);
        for (size_t i = 0; i < n; ++i) keep[i] = b->ctx[i]->launches;
        capture_batch(*b, *params);
        for (size_t i = 0; i < n; ++i) b->ctx[i]->launches = keep[i];
      }
    }
    for (Ctx* c : b->ctx)
      VLB_CUDA(cudaMemcpyAsync(c->hsc, c->dsc, sizeof(DeviceScalars), cudaMemcpyDeviceToHost, b->origin));
    VLB_CUDA(cudaEventRecord(b->fork, b->origin));
    for (Ctx* c : b->ctx) VLB_CUDA(cudaStreamWaitEvent(c->stream, b->fork, 0));  // later work on a context follows
    VLB_CUDA(cudaStreamSynchronize(b->origin));
    int rc = VLB_OK;
    for (size_t i = 0; i < n; ++i) {
      Ctx& c = *b->ctx[i];
      collect_step(c, projs ? &projs[i] : nullptr, params, results ? &results[i] : nullptr);
      if (int r = status_code(c)) rc = r;
    }
    return rc;
  });
}

int vlb_exchange_buffers(vlb_ctx* ctx, int32_t deposit_mode, vlb_exchange* out) {
  CTX_OR_FAIL;
  if (!out) return fail(VLB_ERR_ARG, "null exchange descriptor");
  if (deposit_mode != VLB_DEPOSIT_FLOAT32 && deposit_mode != VLB_DEPOSIT_FIXED64)
    return fail(VLB_ERR_ARG, "unknown deposit mode");
  const int64_t nf = (int64_t)c.fine.n * c.fine.n * c.fine.n, nc = (int64_t)c.coarse.n * c.coarse.n * c.coarse.n;
  *out = vlb_exchange{};
  if (deposit_mode == VLB_DEPOSIT_FIXED64) {
    out->rho_fine = c.rho_fixed;
    out->rho_fine_dtype = VLB_DTYPE_INT64;
  } else {
    out->rho_fine = c.fine.rho;
    out->rho_fine_dtype = VLB_DTYPE_FLOAT32;
  }
  out->rho_fine_count = nf;
  if (deposit_mode == VLB_DEPOSIT_FIXED64) {
    out->rho_coarse = c.rho_fixed_c;
    out->rho_coarse_dtype = VLB_DTYPE_INT64;
  } else {
    out->rho_coarse = c.coarse.rho;
    out->rho_coarse_dtype = VLB_DTYPE_FLOAT32;
  }
  out->rho_coarse_count = nc;
  out->scalars = c.dsc->xch;
  out->scalars_count = 1;
  out->reaction = c.dsc->red;
  out->reaction_count = 4;
  out->stream = c.stream;
  return VLB_OK;
}

int vlb_step_deposit(vlb_ctx* ctx, const vlb_projectile* proj, const vlb_step_params* params) {
  CTX_OR_FAIL;
  if (int rc = check_step_params(c, params)) return rc;
  if (params->film) return fail(VLB_ERR_ARG, "a sharded step takes no film frames (params.film must be 0)");
  c.mode_precision = params->poisson_precision;
  return guarded([&]() -> int {
    upload_projectile(c, proj);
    enqueue_phase_deposit(c, *params, 0);
    c.shard_phase = 1;
    return VLB_OK;
  });
}

int vlb_step_fields(vlb_ctx* ctx, const vlb_step_params* params, int64_t npart_global) {
  CTX_OR_FAIL;
  if (int rc = check_step_params(c, params)) return rc;
  if (c.shard_phase != 1) return fail(VLB_ERR_STATE, "vlb_step_fields before vlb_step_deposit");
  if (npart_global < c.N) return fail(VLB_ERR_ARG, "the whole cloud cannot be smaller than this shard");
  c.mode_precision = params->poisson_precision;
  return guarded([&]() -> int {
    enqueue_phase_fields(c, *params, npart_global);
    c.shard_phase = 2;
    return VLB_OK;
  });
}

int vlb_step_advance(vlb_ctx* ctx, vlb_projectile* proj, const vlb_step_params* params, vlb_step_result* result) {
  CTX_OR_FAIL;
  if (int rc = check_step_params(c, params)) return rc;
  if (c.shard_phase != 2) return fail(VLB_ERR_STATE, "vlb_step_advance before vlb_step_fields");
  return guarded([&]() -> int {
    enqueue_phase_advance(c, *params);
    c.shard_phase = 0;
    finish_step(c, proj, params, result);
    return status_code(c);
  });
}

int vlb_get_grid(vlb_ctx* ctx, int32_t which, float* host) {
  CTX_OR_FAIL;
  if (!host) return fail(VLB_ERR_ARG, "null host buffer");
  return guarded([&]() -> int {
    float* g = grid_ptr(c, which);
    VLB_CUDA(cudaMemcpyAsync(host, g, grid_size(c, which) * 4, cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_set_grid(vlb_ctx* ctx, int32_t which, const float* host) {
  CTX_OR_FAIL;
  if (!host) return fail(VLB_ERR_ARG, "null host buffer");
  return guarded([&]() -> int {
    float* g = grid_ptr(c, which);
    VLB_CUDA(cudaMemcpyAsync(g, host, grid_size(c, which) * 4, cudaMemcpyHostToDevice, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_get_forces(vlb_ctx* ctx, float* host) {
  CTX_OR_FAIL;
  if (!host) return fail(VLB_ERR_ARG, "null host buffer");
  return guarded([&]() -> int {
    const size_t n = (size_t)c.N;
    for (int a = 0; a < 3; ++a)
      VLB_CUDA(cudaMemcpyAsync(host + a * n, c.force + a * c.Npad, n * 4, cudaMemcpyDeviceToHost, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_set_forces(vlb_ctx* ctx, const float* host) {
  CTX_OR_FAIL;
  if (!host) return fail(VLB_ERR_ARG, "null host buffer");
  return guarded([&]() -> int {
    const size_t n = (size_t)c.N;
    for (int a = 0; a < 3; ++a)
      VLB_CUDA(cudaMemcpyAsync(c.force + a * c.Npad, host + a * n, n * 4, cudaMemcpyHostToDevice, c.stream));
    VLB_CUDA(cudaStreamSynchronize(c.stream));
    return VLB_OK;
  });
}

int vlb_enclosed_charge(vlb_ctx* ctx, const double position[3], double radius, double* q) {
  CTX_OR_FAIL;
  if (!position || !q) return fail(VLB_ERR_ARG, "null argument");
  return guarded([&]() -> int {
    vlb_projectile p{};
    for (int d = 0; d < 3; ++d) p.position[d] = position[d];
    upload_projectile(c, &p);
    launch_enclosed(c, radius);
    fetch_scalars(c);
    *q = c.weight * (double)c.hsc->enclosed;
    return VLB_OK;
  });
}

int vlb_profile(vlb_ctx* ctx, int32_t enable) {
  CTX_OR_FAIL;
  c.profile = enable != 0;
  for (double& m : c.stage_ms) m = 0;
  return VLB_OK;
}

int vlb_stage_count(void) { return kEvGatherBegin + 1; }

const char* vlb_stage_name(int32_t i) { return (i >= 0 && i < kNumStages) ? kStageNames[i] : ""; }

int vlb_stage_times(vlb_ctx* ctx, double* ms, int32_t n) {
  CTX_OR_FAIL;
  if (!ms) return fail(VLB_ERR_ARG, "null output");
  for (int i = 0; i < std::min<int>(n, kNumStages); ++i) ms[i] = c.stage_ms[i];
  return VLB_OK;
}

int vlb_launch_count(vlb_ctx* ctx, int64_t* count) {
  CTX_OR_FAIL;
  if (!count) return fail(VLB_ERR_ARG, "null output");
  *count = c.launches;
  return VLB_OK;
}

int vlb_fp32_peak(int32_t device, double* tflops) {
  if (!tflops) return fail(VLB_ERR_ARG, "null output");
  return guarded([&]() -> int {
    *tflops = measure_fp32_peak(device);
    return VLB_OK;
  });
}

int vlb_stream(vlb_ctx* ctx, void** stream) {
  CTX_OR_FAIL;
  if (!stream) return fail(VLB_ERR_ARG, "null output");
  *stream = (void*)c.stream;
  return VLB_OK;
}

}  // extern "C"
