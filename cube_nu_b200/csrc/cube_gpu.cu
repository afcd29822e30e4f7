// C ABI and step orchestration for one CUBE image on one B200.
//
// Replaces the reference's zero-argument step subroutines (main.f90:33-38; drift.f90,
// kick.f90, particle_mesh.f90) with explicit calls on a context that owns the
// device-resident particle state between cube_gpu_upload and cube_gpu_download.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/cube_gpu.h"
#include "common.cuh"
#include "fft.cuh"
#include "fft2.cuh"
#include "kernels.cuh"
#include "ic.cuh"
#include "power.cuh"
#include "pp.cuh"
#include "dpm.cuh"
#include "slab.cuh"

using namespace cube;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(CUBE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

bool smooth23(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

struct FFTTable {
  int n = 0;
  float2* tw = nullptr;
  FFTDesc desc;
};

// Kernel classes for the opt-in event timers (cube_gpu_profile).
enum KClass {
  K_DRIFT_DEST, K_DRIFT_SCATTER, K_DRIFT_SORT, K_DRIFT_GATHER, K_SCAN, K_DEP_PM1, K_FFT_PM1, K_F2_PM1, K_INT_PM1,
  K_DEP_PM2, K_FFTX_PM2, K_FFTY_PM2, K_FFTZ_PM2, K_FFTC_PM2, K_F2_PM2, K_INT_PM2, K_DEP_PM3, K_FFTX_PM3, K_FFTY_PM3,
  K_FFTZ_PM3, K_FFTC_PM3, K_F2_PM3, K_INT_PM3, K_PP, K_CLASSIFY, K_GREEN, K_FILL, K_PK_DEP, K_PK_FFT, K_PK_BIN,
  K_PK_ALIAS, K_MOMENTUM, K_MASS, K_SLAB, K_NCLASS
};
const char* const KNAMES[K_NCLASS] = {
    "drift_dest", "drift_scatter", "drift_sort", "drift_gather", "scan", "deposit_pm1", "fft_pm1", "f2max_pm1",
    "interp_pm1", "deposit_pm2", "fft_x_pm2", "fft_y_pm2", "fft_z_green_pm2", "fft_c2r_pm2", "f2max_pm2",
    "interp_pm2", "deposit_pm3", "fft_x_pm3", "fft_y_pm3", "fft_z_green_pm3", "fft_c2r_pm3", "f2max_pm3",
    "interp_pm3", "pp", "classify", "green", "fill_pcell", "pk_deposit", "pk_fft", "pk_bin", "pk_alias", "momentum", "mass_pm3",
    "slab_exchange"};

struct ProfRec {
  int cls;
  int a, b;  // event pool indices
};

// Results of a step that the host reads back with one copy at its end.
struct StepRes {
  float red[64];  // f2max[4] (pm1, pm2, pm3, pp), vmax[3][3] at 8.. (pm2, pm3, pp)
  unsigned long long pairs, cand;  // PP pairs within range, PP candidate pairs
  unsigned err;       // device error word (CUBE_DEVERR_*)
  unsigned overflow;  // a PM3 class outgrew the captured plan
  int32_t napm[8];
  int32_t maxcount;   // largest coarse-cell occupancy (PP tuning class)
  int32_t pad;
  int64_t total;      // particles placed by the drift
  unsigned long long msum[3 * MASS_SLOTS * MASS_STRIDE];
  double mom[3 * MOM_BLOCKS];
};

// Shape of the queue PP (pp.cuh): light-cell threshold T, items of B particles (the heavy
// kernel's block), candidate chunks of J particles in shared memory.
struct PPShape {
  int T = 64, B = 256, J = 512;
  bool operator==(const PPShape& o) const { return T == o.T && B == o.B && J == o.J; }
};

// PP tuning classes by the largest cell occupancy.
int pp_class(int maxcount) { return maxcount <= 64 ? 0 : maxcount <= 512 ? 1 : maxcount <= 4096 ? 2 : 3; }

// One captured step (drift + kick) as an executable CUDA graph, for one particle-buffer
// parity, particle count, PM3 plan and PP shape.
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  int parity = 0;
  int64_t np = 0;
  PM3Plan plan;
  PPShape pps;
  bool prof = false;
  int64_t kernels = 0;                 // kernel launches in one replay
  std::vector<cudaEvent_t> events;     // per-kernel timer events recorded by the graph
  std::vector<ProfRec> recs;
};

bool same_plan(const PM3Plan& a, const PM3Plan& b) {
  if (a.nk != b.nk || a.per_max != b.per_max) return false;
  for (int i = 2; i <= 5; ++i)
    if (a.cap[i] != b.cap[i] || a.per[i] != b.per[i] || a.kbase[i] != b.kbase[i] || a.skip[i] != b.skip[i])
      return false;
  return true;
}

}  // namespace

struct cube_ctx {
  cube_params P;
  Geo G;
  int device = 0;
  cudaStream_t s = nullptr;
  int nsm = 148;  // multiprocessors of the device
  bool loaded = false;
  int64_t np = 0, cap = 0;
  int xbytes = 1;
  int ns3 = 0, ntiles = 0;
  // particles (current and drift output)
  void *xp = nullptr, *xp2 = nullptr;
  float *vp = nullptr, *vp2 = nullptr;
  int64_t *pid = nullptr, *pid2 = nullptr;
  int32_t *pcell = nullptr, *pcell2 = nullptr;
  // cells
  int32_t *rhoc = nullptr, *rhoc2 = nullptr, *fill = nullptr, *biglist = nullptr, *nbig = nullptr;
  int32_t* hugelist = nullptr;  // segments beyond the shared-memory sorter; nbig[1] counts them
  int64_t *cstart = nullptr, *cstart2 = nullptr, *scan_tmp = nullptr;
  // drift scratch
  int32_t* dest = nullptr;
  uint64_t *key = nullptr, *skey = nullptr;
  uint32_t* ssrc = nullptr;
  // step results (device) and their pinned host copy; the pointers below point into rdev:
  // reductions f2max[4] (pm1, pm2, pm3, pp) and vmax[3][3] (pm2, pm3, pp); FP64 mass sums
  // [level 1..3][MASS_SLOTS] (int64 or double by deposit form); momentum partials
  // [MOM_BLOCKS][3]; the error word, class histogram, drift total and plan overflow flag
  StepRes* rdev = nullptr;
  StepRes* rhost = nullptr;
  float* red = nullptr;
  unsigned long long* pairs = nullptr;  // pairs[0] in range, pairs[1] candidates
  unsigned long long* msum = nullptr;
  double* mom = nullptr;
  unsigned* err = nullptr;
  unsigned* overflow = nullptr;
  int32_t* napm = nullptr;
  int64_t* total = nullptr;
  int32_t* ires = nullptr;
  int32_t* h_ires = nullptr;  // pinned
  // per-step scalars (device) and their pinned host staging copy
  StepDev* sd = nullptr;
  StepDev* h_sd = nullptr;
  // PM3 class lists: box_slot [nk][ns3], box_sub [nk][per_max]
  int32_t* box_slot = nullptr;
  int32_t* box_sub = nullptr;
  int64_t slot_cap = 0, sub_cap = 0;  // allocated entries
  // captured steps (cube_params.step_graph)
  std::vector<StepGraph> graphs;
  StepGraph* cap_graph = nullptr;  // the graph being captured (timers and launches go to it)
  int32_t napm_est[8] = {0};       // class histogram of the last step (plan of the next capture)
  bool have_est = false;
  int32_t maxcount_est = -1;       // largest cell occupancy of the last step (-1: unknown)
  // queue PP (cube_params.pp_queue): decoded offsets, heavy-cell list and item prefix,
  // queue counters; the autotuner's scratch velocities and reductions, and its winners
  float4* pfin = nullptr;
  int32_t* hperm = nullptr;  // heavy cells' particles ordered by neighbour-set code (pp.cuh)
  int32_t* hlist = nullptr;
  int* hpre = nullptr;
  int* ppq = nullptr;
  float* vtune = nullptr;
  float* tune_red = nullptr;  // f2max, vmax[3] at 8, pairs (u64) at 16
  PPShape pp_best[4];
  bool pp_tuned[4] = {false, false, false, false};
  double pp_tune_ms[4] = {0, 0, 0, 0};
  void* xp_base = nullptr;         // parity of the particle buffers: xp == xp_base or not
  // meshes
  void* arena = nullptr;
  size_t arena_bytes = 0;
  float* green1 = nullptr;
  float* green2 = nullptr;
  // neutrino linear response: force kernels tf = interp_tf_F(|k|) * Gk per level (or
  // (1 - f_nu) * Gk without a table), rebuilt in place when the table changes
  float* tf1 = nullptr;
  float* tf2 = nullptr;
  float* tf3[8] = {nullptr};
  int tf_ver[10] = {0};       // table version each kernel was built from (1, 2, 3 + class)
  float* nu_tab = nullptr;    // log k [nb] then log tf_F [nb]
  int nu_nb = 0, nu_ver = 1;
  float* green3[8] = {nullptr};
  std::vector<FFTTable> ffts;
  // capture for tests
  int cap_level = 0, cap_box = -1, cap_what = -1;
  float* cap_buf = nullptr;
  int64_t cap_n = 0;
  // timing
  cudaEvent_t ev[8];
  // asynchronous checkpoint: side stream, staging copies in pinned memory, the event that
  // marks the copies done, and the writer thread with its status
  cudaStream_t s3 = nullptr;
  cudaEvent_t ev_ckpt = nullptr;
  bool ckpt_pending = false;
  void* ck_host = nullptr;
  size_t ck_bytes = 0;
  std::thread ck_thread;
  int ck_status = 0;
  std::string ck_error;
  // side stream of cube_gpu_step_host (copies that overlap the step), created at first use
  cudaStream_t s2 = nullptr;
  cudaEvent_t ev_up = nullptr, ev_drift = nullptr;
  // 1: use the generic Stockham passes for every size (CUBE_FFT_GENERIC=1)
  int fft_generic = 0;
  // 1: fused plane FFT kernels for sides <= 144 (CUBE_FFT_FUSED, default 1)
  int fft_fused = 1;
  // opt-in per-kernel timers and the launch counter
  bool prof = false;
  std::vector<cudaEvent_t> pool;
  int pool_used = 0;
  std::vector<ProfRec> pending;
  double prof_ms[K_NCLASS] = {0};
  int64_t prof_n[K_NCLASS] = {0};
  int64_t launches = 0;
  // a run split into z-slabs (cube_params.nslab > 1): the host's collectives; whether the
  // store holds fresh ghost layers; this rank's particles [own0, own1) in the store;
  // scratch of the layer exchange (counts and their prefixes: send down, send up, from
  // below, from above; payloads)
  cube_comm comm{};
  bool have_comm = false;
  bool ghosts = false;
  int64_t own0 = 0, own1 = 0;
  int32_t* lay_cnt = nullptr;
  int64_t* lay_start = nullptr;
  char* lay_buf = nullptr;
  size_t lay_bytes = 0;
};

namespace {

int pool_event(cube_ctx* c) {
  if (c->pool_used == (int)c->pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->pool.push_back(e);
  }
  return c->pool_used++;
}

// Timer events: during a capture they come from the graph's own list and are recorded as
// graph event nodes (cudaEventRecordExternal); otherwise from the context pool.
int timer_event(cube_ctx* c) {
  if (c->cap_graph) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->cap_graph->events.push_back(e);
    return (int)c->cap_graph->events.size() - 1;
  }
  return pool_event(c);
}

void record_timer(cube_ctx* c, int i) {
  if (c->cap_graph) cudaEventRecordWithFlags(c->cap_graph->events[i], c->s, cudaEventRecordExternal);
  else cudaEventRecord(c->pool[i], c->s);
}

// A context event (ev[]) marking a stage boundary; a graph event node while capturing.
cudaError_t mark(cube_ctx* c, cudaEvent_t e) {
  return c->cap_graph ? cudaEventRecordWithFlags(e, c->s, cudaEventRecordExternal) : cudaEventRecord(e, c->s);
}

void prof_begin(cube_ctx* c, int cls, int nlaunch, int& a) {
  if (c->cap_graph) c->cap_graph->kernels += nlaunch;
  else c->launches += nlaunch;
  a = -1;
  if (!c->prof) return;
  a = timer_event(c);
  record_timer(c, a);
  (void)cls;
}

void prof_end(cube_ctx* c, int cls, int a) {
  if (!c->prof || a < 0) return;
  const int b = timer_event(c);
  record_timer(c, b);
  if (c->cap_graph) c->cap_graph->recs.push_back({cls, a, b});
  else c->pending.push_back({cls, a, b});
}

// After a stream synchronisation: fold the pending event pairs into the totals.
void prof_collect(cube_ctx* c) {
  for (const ProfRec& r : c->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->pool[r.a], c->pool[r.b]) == cudaSuccess) {
      c->prof_ms[r.cls] += ms;
      c->prof_n[r.cls] += 1;
    }
  }
  c->pending.clear();
  c->pool_used = 0;
}

#define LAUNCH(c, cls, nl, ...)     \
  do {                              \
    int a_;                         \
    prof_begin((c), (cls), (nl), a_); \
    __VA_ARGS__;                    \
    prof_end((c), (cls), a_);       \
  } while (0)

const FFTDesc* fft_desc(cube_ctx* c, int n) {
  for (auto& t : c->ffts)
    if (t.n == n) return &t.desc;
  return nullptr;
}

int add_fft(cube_ctx* c, int n) {
  if (fft_desc(c, n)) return 0;
  if (!smooth23(n)) return fail(CUBE_E_ARG, "FFT size " + std::to_string(n) + " is not of the form 2^a 3^b");
  FFTTable t;
  t.n = n;
  std::vector<float2> h(n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  CK(cudaMalloc(&t.tw, n * sizeof(float2)));
  CK(cudaMemcpy(t.tw, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  t.desc.n = n;
  t.desc.tw = t.tw;
  int m = n, k = 0;
  while (m % 4 == 0 && k < 15) { t.desc.rad[k++] = 4; m /= 4; }
  while (m % 2 == 0 && k < 15) { t.desc.rad[k++] = 2; m /= 2; }
  while (m % 3 == 0 && k < 15) { t.desc.rad[k++] = 3; m /= 3; }
  if (m != 1) return fail(CUBE_E_ARG, "FFT size too large");
  t.desc.nrad = k;
  c->ffts.push_back(t);
  return 0;
}

Geo make_geo(const cube_params& p) {
  Geo g;
  memset(&g, 0, sizeof(g));
  g.ng = (int)p.ng;
  g.rcs = (int)p.ratio_cs;
  g.nnt = (int)p.nnt;
  g.nns = (int)p.nns;
  g.ncb = (int)p.ncb;
  g.ngb = (int)p.ngb;
  g.nc = g.ng / g.rcs;
  g.nt = g.nc / g.nnt;
  g.ntt = g.nt / g.nns;
  g.ngp = g.ng / g.nnt;
  g.ngt = g.ngp + 2 * g.ngb;
  g.izipx = p.izipx;
  for (int i = 1; i <= 7; ++i) {
    g.nfp[i] = (g.ngp / g.nns) * rsf_of(i);
    g.nfb[i] = g.rcs * rsf_of(i);
    g.nft[i] = g.nfp[i] + 2 * g.nfb[i];
  }
  g.app = p.app;
  g.apm1c = p.apm1c;
  g.apm2 = p.apm2;
  g.apm3f = p.apm3f;
  g.mass_p = p.mass_p_cdm;
  g.f_nu = p.f_nu;
  g.x_res = std::ldexp(1.0, -8 * g.izipx);
  g.inv_step = 1.0 / (g.x_res * (double)g.rcs);
  g.zmask = (g.izipx == 1) ? 0xffu : 0xffffu;
  g.ncells = (int64_t)g.nc * g.nc * g.nc;
  // this context's slab: tile layers [slab*L, (slab+1)*L) along z, L = nnt/nslab
  g.nslab = p.nslab > 1 ? p.nslab : 1;
  const int L = g.nnt / g.nslab, slab = g.nslab > 1 ? p.slab : 0;
  g.tile0 = slab * L * g.nnt * g.nnt;
  g.tile1 = (slab + 1) * L * g.nnt * g.nnt;
  g.s0 = g.tile0 * g.nns * g.nns * g.nns;
  g.s1 = g.tile1 * g.nns * g.nns * g.nns;
  g.c0 = (int64_t)g.tile0 * g.nt * g.nt * g.nt;
  g.c1 = (int64_t)g.tile1 * g.nt * g.nt * g.nt;
  return g;
}

// In-place mesh layouts (fft2.cuh): boxes of side n are n planes of `psb` bytes.
//  row-pitched: rows of RP = max(n*rb, (n/2+1)*8) bytes, psb = n*RP;
//  plane-compact (sizes that run the fused plane FFT): rows of n reals / n/2+1 complex /
//    n floats from the start of the plane, psb = max(n*n*rb, n*(n/2+1)*8).
// rb = 4, or 8 for the int64 fixed-point deposit.
struct Pitch {
  int64_t rp;    // bytes per real row (capture copies)
  int64_t psb;   // bytes per plane
  int pr, pc, pf;        // row pitch: real elements, complex elements, floats
  int64_t plr, plc, plf;  // plane pitch in the same units
};

bool fused_layout(const cube_ctx* c, int n);

Pitch pitch_of(const cube_ctx* c, int n, bool fixed) {
  const int64_t rb = fixed ? 8 : 4, nh = n / 2 + 1;
  Pitch p;
  if (fused_layout(c, n)) {
    p.psb = std::max<int64_t>((int64_t)n * n * rb, (int64_t)n * nh * 8);
    p.pr = n;
    p.pc = (int)nh;
    p.pf = n;
    p.rp = n * rb;
  } else {
    p.rp = std::max<int64_t>((int64_t)n * rb, nh * 8);
    p.psb = n * p.rp;
    p.pr = (int)(p.rp / rb);
    p.pc = (int)(p.rp / 8);
    p.pf = (int)(p.rp / 4);
  }
  p.plr = p.psb / rb;
  p.plc = p.psb / 8;
  p.plf = p.psb / 4;
  return p;
}

size_t mesh_bytes(const cube_ctx* c, int n, int64_t nbox, bool fixed) {
  return (size_t)nbox * n * pitch_of(c, n, fixed).psb + 256;
}

struct MeshPtrs {
  void* real;
  float2* ck;
  Pitch pt;
};
MeshPtrs mesh_ptrs(cube_ctx* c, int n, int64_t, bool fixed) {
  MeshPtrs m;
  m.real = c->arena;
  m.ck = reinterpret_cast<float2*>(c->arena);
  m.pt = pitch_of(c, n, fixed);
  return m;
}

// The owner-computes PM3 deposit covers a class when every region of DEP3_R x DEP3_R x
// DEP3_RZ cells of its boxes draws on at most DEP3_MAXC coarse cells (same range as
// dep3_krange).
bool dep3_own_fits(const Geo& G, int iapm) {
  const int nft = G.nft[iapm], nfb = G.nfb[iapm];
  auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
  auto most = [&](int R) {
    int mk = 0;
    for (int o = 0; o < nft; o += R) {
      const int e = std::min(R, nft - o);
      const int klo = std::max(-1, fdiv(o - nfb - 2, nfb)), khi = std::min(G.ntt, fdiv(o + e - nfb + 1, nfb));
      mk = std::max(mk, khi - klo + 1);
    }
    return (int64_t)mk;
  };
  return nfb > 0 && most(DEP3_R) * most(DEP3_R) * most(DEP3_RZ) <= DEP3_MAXC;
}

// How many boxes of side n fit in the arena.
int64_t boxes_fit(cube_ctx* c, int n, bool fixed) {
  const size_t per = mesh_bytes(c, n, 1, fixed);
  return std::max<int64_t>(1, (int64_t)(c->arena_bytes / per));
}

// Raise a kernel's dynamic shared-memory limit when `bytes` plus its static shared memory
// pass the 48 KB default and the limit set so far is lower.
template <typename K>
void smem_optin(K kernel, size_t bytes) {
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, kernel) != cudaSuccess) return;
  if (bytes + a.sharedSizeBytes > 48 * 1024 && bytes > (size_t)a.maxDynamicSharedSizeBytes)
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Size-specialised passes (fft2.cuh) for N = R1*R2.  N <= 144 runs the fused plane
// kernels (XY forward, YX inverse) around the z pass; larger N runs five passes.
// z pass with Green multiply for the row-pitched sizes (N >= 192): the persistent
// streamed kernel, which keeps the next line's loads in flight.
template <int N, int R1, int R2>
void fz_green(cube_ctx* c, int64_t nbox, float2* ck, const float* green, const float2* tw, const Pitch& pt, int kz) {
  constexpr int T = f2::TPS<R1, R2>::T;
  int W = 0, ncg = 0;
  f2::fz_stream_shape(N, T, W, ncg);
  const size_t sm = f2::fz_stream_smem(N, W);
  const int64_t nitems = nbox * (int64_t)N * ncg;
  const unsigned grid = (unsigned)std::min<int64_t>(nitems, 2 * (int64_t)c->nsm);
  smem_optin(f2::k_fz_stream<N, R1, R2>, sm);
  LAUNCH(c, kz, 1, f2::k_fz_stream<N, R1, R2><<<grid, W * T, sm, c->s>>>(ck, green, tw, W, ncg, pt.pc, pt.plc, nitems));
}

template <int N, int R1, int R2>
void fft2_run(cube_ctx* c, int64_t nbox, const void* real_in, bool fixed, float scale, float* phi_out, float2* ck,
              const float* green, float inv, int kx, int ky, int kz, int kc, const Pitch& pt) {
  constexpr int T = f2::TPS<R1, R2>::T, NH = N / 2 + 1;
  const float2* tw = fft_desc(c, N)->tw;
  const int64_t nrows = nbox * (int64_t)N * N;
  const int W = f2::fcol_width(N, T);
  const size_t smc = (size_t)(N + W * N) * sizeof(float2);
  dim3 gc((unsigned)(nbox * N), (unsigned)((NH + W - 1) / W));
  if constexpr (N <= 144) {
    if (fused_layout(c, N)) {
      const size_t smf = f2::Plane3Sm<N>::FWD, smi = f2::Plane3Sm<N>::INV;
      const unsigned planes = (unsigned)(nbox * N);
      if (fixed) {
        smem_optin(f2::k_fxy3_r2c<N, R1, R2, long long>, smf);
        LAUNCH(c, kx, 1, f2::k_fxy3_r2c<N, R1, R2, long long><<<planes, f2::PLANE3_THREADS, smf, c->s>>>(
                             (const long long*)real_in, ck, tw, scale, pt.pr, pt.pc, pt.plr, pt.plc));
      } else {
        smem_optin(f2::k_fxy3_r2c<N, R1, R2, float>, smf);
        LAUNCH(c, kx, 1, f2::k_fxy3_r2c<N, R1, R2, float><<<planes, f2::PLANE3_THREADS, smf, c->s>>>(
                             (const float*)real_in, ck, tw, scale, pt.pr, pt.pc, pt.plr, pt.plc));
      }
      // plane sizes: the block-per-line column pass hides latency with more warps
      const size_t smg = smc + (size_t)W * N * sizeof(float);  // + prefetched Green values
      smem_optin(f2::k_fcol3<N, R1, R2, 2, 2>, smg);
      LAUNCH(c, kz, 1, f2::k_fcol3<N, R1, R2, 2, 2><<<gc, W * T, smg, c->s>>>(ck, green, tw, W, pt.pc, pt.plc));
      smem_optin(f2::k_fyx3_c2r<N, R1, R2>, smi);
      LAUNCH(c, kc, 1, f2::k_fyx3_c2r<N, R1, R2><<<planes, f2::PLANE3_THREADS, smi, c->s>>>(
                           ck, phi_out, tw, inv, pt.pc, pt.pf, pt.plc, pt.plf));
      return;
    }
  }
  const int S = std::max(1, 256 / T);
  const size_t smx = (size_t)(N + S * N) * sizeof(float2);
  const unsigned gx = (unsigned)((nrows + 2 * S - 1) / (2 * S));
  if (fixed) {
    smem_optin(f2::k_fx_r2c<N, R1, R2, long long>, smx);
    LAUNCH(c, kx, 1, f2::k_fx_r2c<N, R1, R2, long long><<<gx, S * T, smx, c->s>>>((const long long*)real_in, ck, nrows,
                                                                                 tw, scale, pt.pr, pt.pc));
  } else {
    smem_optin(f2::k_fx_r2c<N, R1, R2, float>, smx);
    LAUNCH(c, kx, 1, f2::k_fx_r2c<N, R1, R2, float><<<gx, S * T, smx, c->s>>>((const float*)real_in, ck, nrows, tw,
                                                                             scale, pt.pr, pt.pc));
  }
  smem_optin(f2::k_fcol3<N, R1, R2, 1, 0>, smc);
  smem_optin(f2::k_fcol3<N, R1, R2, 1, 1>, smc);
  smem_optin(f2::k_fx_c2r<N, R1, R2>, smx);
  LAUNCH(c, ky, 1, f2::k_fcol3<N, R1, R2, 1, 0><<<gc, W * T, smc, c->s>>>(ck, nullptr, tw, W, pt.pc, pt.plc));
  fz_green<N, R1, R2>(c, nbox, ck, green, tw, pt, kz);
  LAUNCH(c, ky, 1, f2::k_fcol3<N, R1, R2, 1, 1><<<gc, W * T, smc, c->s>>>(ck, nullptr, tw, W, pt.pc, pt.plc));
  LAUNCH(c, kc, 1, f2::k_fx_c2r<N, R1, R2><<<gx, S * T, smx, c->s>>>(ck, phi_out, nrows, tw, inv, pt.pc, pt.pf));
}

bool fft2_size(int n) {
  switch (n) {
    case 16: case 32: case 48: case 64: case 96: case 128: case 144: case 192: case 256: case 288: case 432:
    case 512: case 576: case 1024:
      return true;
    default:
      return false;
  }
}

bool fused_layout(const cube_ctx* c, int n) { return !c->fft_generic && c->fft_fused && n <= 144 && fft2_size(n); }

bool fft2_dispatch(cube_ctx* c, int n, int64_t nbox, const void* real_in, bool fixed, float scale, float* phi_out,
                   float2* ck, const float* green, float inv, int kx, int ky, int kz, int kc, const Pitch& pt) {
#define CUBE_FFT2(N, R1, R2) \
  case N: fft2_run<N, R1, R2>(c, nbox, real_in, fixed, scale, phi_out, ck, green, inv, kx, ky, kz, kc, pt); return true;
  switch (n) {
    CUBE_FFT2(16, 4, 4)
    CUBE_FFT2(32, 4, 8)
    CUBE_FFT2(48, 8, 6)
    CUBE_FFT2(64, 8, 8)
    CUBE_FFT2(96, 8, 12)
    CUBE_FFT2(128, 8, 16)
    CUBE_FFT2(144, 12, 12)
    CUBE_FFT2(192, 16, 12)
    CUBE_FFT2(256, 16, 16)
    CUBE_FFT2(288, 16, 18)
    CUBE_FFT2(432, 24, 18)
    CUBE_FFT2(512, 16, 32)
    CUBE_FFT2(576, 24, 24)
    CUBE_FFT2(1024, 32, 32)
    default: return false;
  }
#undef CUBE_FFT2
}

// Forward-only r2c transform of one real mesh (float, layout of pitch_of(c, N, false))
// into its half spectrum, in place: the x (or fused xy) pass, then y and z forward.
template <int N, int R1, int R2>
void fft2_forward(cube_ctx* c, float* real, const Pitch& pt, int cls) {
  constexpr int T = f2::TPS<R1, R2>::T, NH = N / 2 + 1;
  const float2* tw = fft_desc(c, N)->tw;
  float2* ck = reinterpret_cast<float2*>(real);
  const int64_t nrows = (int64_t)N * N;
  const int W = f2::fcol_width(N, T);
  const size_t smc = (size_t)(N + W * N) * sizeof(float2);
  dim3 gc((unsigned)N, (unsigned)((NH + W - 1) / W));
  smem_optin(f2::k_fcol3<N, R1, R2, 2, 0>, smc);
  if constexpr (N <= 144) {
    if (fused_layout(c, N)) {
      const size_t smf = f2::Plane3Sm<N>::FWD;
      smem_optin(f2::k_fxy3_r2c<N, R1, R2, float>, smf);
      LAUNCH(c, cls, 1, f2::k_fxy3_r2c<N, R1, R2, float><<<(unsigned)N, f2::PLANE3_THREADS, smf, c->s>>>(
                            real, ck, tw, 1.f, pt.pr, pt.pc, pt.plr, pt.plc));
      LAUNCH(c, cls, 1, f2::k_fcol3<N, R1, R2, 2, 0><<<gc, W * T, smc, c->s>>>(ck, nullptr, tw, W, pt.pc, pt.plc));
      return;
    }
  }
  const int S = std::max(1, 256 / T);
  const size_t smx = (size_t)(N + S * N) * sizeof(float2);
  const unsigned gx = (unsigned)((nrows + 2 * S - 1) / (2 * S));
  smem_optin(f2::k_fx_r2c<N, R1, R2, float>, smx);
  smem_optin(f2::k_fcol3<N, R1, R2, 1, 0>, smc);
  LAUNCH(c, cls, 1, f2::k_fx_r2c<N, R1, R2, float><<<gx, S * T, smx, c->s>>>(real, ck, nrows, tw, 1.f, pt.pr, pt.pc));
  LAUNCH(c, cls, 1, f2::k_fcol3<N, R1, R2, 1, 0><<<gc, W * T, smc, c->s>>>(ck, nullptr, tw, W, pt.pc, pt.plc));
  LAUNCH(c, cls, 1, f2::k_fcol3<N, R1, R2, 2, 0><<<gc, W * T, smc, c->s>>>(ck, nullptr, tw, W, pt.pc, pt.plc));
}

// Forward-only r2c with the generic Stockham passes (any 2^a 3^b size, row-pitched layout):
// x r2c, then the column kernel along y and, with the two pitches swapped, along z (the
// plane pitch of the row-pitched layout is n row pitches, so plane z of line y sits at
// y*pc + z*plc either way).
void fft_forward_generic(cube_ctx* c, int n, float* real, const Pitch& pt, int cls) {
  const FFTDesc& D = *fft_desc(c, n);
  float2* ck = reinterpret_cast<float2*>(real);
  const int nh = n / 2 + 1;
  const int64_t nrows = (int64_t)n * n;
  const int rpb = std::max(1, 2048 / n);
  const size_t smx = (size_t)(n + 2 * rpb * n) * sizeof(float2);
  const unsigned gx = (unsigned)((nrows + rpb - 1) / rpb);
  LAUNCH(c, cls, 1, k_fft_x_r2c<float><<<gx, 256, smx, c->s>>>(real, ck, nrows, D, rpb, 1.f, pt.pr, pt.pc));
  const int W = (n <= 256) ? 16 : (n <= 512 ? 8 : 4);
  const size_t smy = (size_t)(n + 2 * W * n) * sizeof(float2);
  dim3 gy((unsigned)n, (unsigned)((nh + W - 1) / W));
  LAUNCH(c, cls, 1, k_fft_y<<<gy, 256, smy, c->s>>>(ck, D, W, -1, pt.pc, pt.plc));
  LAUNCH(c, cls, 1, k_fft_y<<<gy, 256, smy, c->s>>>(ck, D, W, -1, (int)pt.plc, (int64_t)pt.pc));
}

bool fft2_forward_dispatch(cube_ctx* c, int n, float* real, const Pitch& pt, int cls) {
#define CUBE_FFT2F(N, R1, R2) \
  case N: fft2_forward<N, R1, R2>(c, real, pt, cls); return true;
  switch (n) {
    CUBE_FFT2F(16, 4, 4)
    CUBE_FFT2F(32, 4, 8)
    CUBE_FFT2F(48, 8, 6)
    CUBE_FFT2F(64, 8, 8)
    CUBE_FFT2F(96, 8, 12)
    CUBE_FFT2F(128, 8, 16)
    CUBE_FFT2F(144, 12, 12)
    CUBE_FFT2F(192, 16, 12)
    CUBE_FFT2F(256, 16, 16)
    CUBE_FFT2F(288, 16, 18)
    CUBE_FFT2F(432, 24, 18)
    CUBE_FFT2F(512, 16, 32)
    CUBE_FFT2F(576, 24, 24)
    CUBE_FFT2F(1024, 32, 32)
    default: return false;
  }
#undef CUBE_FFT2F
}

void launch_fft(cube_ctx* c, int n, int64_t nbox, const void* real_in, bool fixed, float scale, float* phi_out,
                float2* ck, const float* green, float norm, int reps, int level) {
  const int kx = level == 1 ? K_FFT_PM1 : level == 2 ? K_FFTX_PM2 : K_FFTX_PM3;
  const int ky = level == 1 ? K_FFT_PM1 : level == 2 ? K_FFTY_PM2 : K_FFTY_PM3;
  const int kz = level == 1 ? K_FFT_PM1 : level == 2 ? K_FFTZ_PM2 : K_FFTZ_PM3;
  const int kc = level == 1 ? K_FFT_PM1 : level == 2 ? K_FFTC_PM2 : K_FFTC_PM3;
  const Pitch pt = pitch_of(c, n, fixed);
  // the backward transform's normalisation (phi/real(nwork)**3, kick.f90:846; PM1 divides
  // by n three times) as one multiplication by the reciprocal, rounded once from double
  const float inv = (float)(1.0 / std::pow((double)norm, (double)reps));
  if (c->fft_generic == 0 &&
      fft2_dispatch(c, n, nbox, real_in, fixed, scale, phi_out, ck, green, inv, kx, ky, kz, kc, pt))
    return;
  const FFTDesc& D = *fft_desc(c, n);
  const int nh = n / 2 + 1;
  const int64_t nrows = nbox * (int64_t)n * n;
  const int rpb = std::max(1, 2048 / n);
  const size_t smx = (size_t)(n + 2 * rpb * n) * sizeof(float2);
  const unsigned gx = (unsigned)((nrows + rpb - 1) / rpb);
  if (fixed)
    LAUNCH(c, kx, 1, k_fft_x_r2c<long long><<<gx, 256, smx, c->s>>>((const long long*)real_in, ck, nrows, D, rpb, scale,
                                                                    pt.pr, pt.pc));
  else
    LAUNCH(c, kx, 1, k_fft_x_r2c<float><<<gx, 256, smx, c->s>>>((const float*)real_in, ck, nrows, D, rpb, scale, pt.pr,
                                                                pt.pc));
  const int W = (n <= 256) ? 16 : (n <= 512 ? 8 : 4);
  const size_t smy = (size_t)(n + 2 * W * n) * sizeof(float2);
  dim3 gy((unsigned)(nbox * n), (unsigned)((nh + W - 1) / W));
  LAUNCH(c, ky, 1, k_fft_y<<<gy, 256, smy, c->s>>>(ck, D, W, -1, pt.pc, pt.plc));
  LAUNCH(c, kz, 1, k_fft_z_green<<<gy, 256, smy, c->s>>>(ck, green, D, W, pt.pc, pt.plc));
  LAUNCH(c, ky, 1, k_fft_y<<<gy, 256, smy, c->s>>>(ck, D, W, +1, pt.pc, pt.plc));
  LAUNCH(c, kc, 1, k_fft_x_c2r<<<gx, 256, smx, c->s>>>(ck, phi_out, nrows, D, rpb, inv, pt.pc, pt.pf));
}

inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

int build_green(cube_ctx* c, float** dst, int n, float soft, float range, float gs) {
  if (*dst) return 0;
  const int64_t m = (int64_t)n * n * (n / 2 + 1);
  CK(cudaMalloc(dst, m * sizeof(float)));
  LAUNCH(c, K_GREEN, 1, k_green<<<nblk(m, 128), 128, 0, c->s>>>(*dst, n, soft, range, gs));
  CK(cudaGetLastError());
  return 0;
}

float* green3(cube_ctx* c, int iapm) {
  const Geo& G = c->G;
  if (build_green(c, &c->green3[iapm], G.nft[iapm], G.apm3f, G.apm2 * (float)rsf_of(iapm), 1.f / (float)rsf_of(iapm)))
    return nullptr;
  return c->green3[iapm];
}

void drop_graphs(cube_ctx* c) {
  if (c->graphs.empty()) return;
  if (c->s) cudaStreamSynchronize(c->s);
  for (auto& g : c->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t e : g.events) cudaEventDestroy(e);
  }
  c->graphs.clear();
}

// The force kernel of a level: the Green table, or with neutrinos (f_nu > 0 or a
// transfer table from cube_gpu_nu_transfer) the rescaled table of kick.f90:23-29,
// rebuilt in place when the transfer table is newer than it (outside any capture: the
// step graph calls this for every level it uses before capturing).
const float* kernel_table(cube_ctx* c, int level, int iapm) {
  const Geo& G = c->G;
  const float* gk = level == 1 ? c->green1 : level == 2 ? c->green2 : green3(c, iapm);
  if (!gk) return nullptr;
  if (!(c->P.f_nu > 0.f) && c->nu_nb < 3) return gk;
  float** tf = level == 1 ? &c->tf1 : level == 2 ? &c->tf2 : &c->tf3[iapm];
  const int n = level == 1 ? G.nc : level == 2 ? G.ngt : G.nft[iapm];
  const int slot = level == 3 ? 3 + iapm : level;
  const int64_t cnt = (int64_t)n * n * (n / 2 + 1);
  if (!*tf) {
    if (cudaMalloc(tf, cnt * sizeof(float)) != cudaSuccess) {
      fail(CUBE_E_CUDA, "out of device memory for a neutrino force kernel");
      return nullptr;
    }
    c->tf_ver[slot] = 0;
  }
  if (c->tf_ver[slot] != c->nu_ver) {
    // box sides of the levels (nu_correction_coarse and nu_correction, power_nu.f90)
    const double size = level == 1 ? (double)c->P.box : level == 2 ? (double)c->P.box / G.nnt
                                                                    : (double)c->P.box / G.nnt / G.nns;
    const int nb = c->nu_nb >= 3 ? c->nu_nb : 0;
    const float scale = (float)(1.0 - (double)c->P.f_nu);
    LAUNCH(c, K_GREEN, 1, k_nu_rescale<<<nblk(cnt), 256, 0, c->s>>>(n, size, gk, *tf, c->nu_tab,
                                                                   c->nu_tab ? c->nu_tab + c->nu_nb : nullptr, nb, scale));
    c->tf_ver[slot] = c->nu_ver;
  }
  return *tf;
}

// Copy a box field (n planes of n rows of n values, row pitch `rp` and plane pitch `psb`
// bytes) into a dense capture buffer when it is the one requested.
void maybe_capture(cube_ctx* c, int level, int64_t box, int what, const void* src, int n, bool fixed_int,
                   int64_t rp, int64_t psb) {
  if (c->cap_level != level || c->cap_box != box || c->cap_what != what) return;
  cudaFree(c->cap_buf);
  c->cap_buf = nullptr;
  const int64_t cnt = (int64_t)n * n * n;
  const size_t eb = fixed_int ? 8 : 4;
  if (cudaMalloc(&c->cap_buf, cnt * eb) != cudaSuccess) return;
  for (int z = 0; z < n; ++z)
    cudaMemcpy2DAsync((char*)c->cap_buf + (size_t)z * n * n * eb, n * eb, (const char*)src + (size_t)z * psb, rp,
                      n * eb, (size_t)n, cudaMemcpyDeviceToDevice, c->s);
  c->cap_n = fixed_int ? -cnt : cnt;  // negative marks int64 content
}

}  // namespace

// =================================================================================
extern "C" {

void cube_params_default(cube_params* p, int64_t ng) {
  memset(p, 0, sizeof(*p));
  p->ng = ng;
  p->ratio_cs = 4;
  p->nnt = 4;
  p->nns = 4;
  p->np_nc = 4;
  p->ncb = 4;
  p->ngb = 16;
  p->izipx = 2;
  p->pm3_on = 1;
  p->pp_on = 1;
  p->deposit_mode = CUBE_DEPOSIT_FP32;
  p->box = 600.f;
  p->app = 0.06f;
  p->apm1c = 3.5f;
  p->apm2 = 3.5f;
  p->apm3f = 3.5f;
  p->mass_p_cdm = 0.f;
  p->nslab = 1;
}

const char* cube_gpu_version(void) { return "cube-b200 0.1 (sm_100a)"; }

int cube_gpu_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return CUBE_E_ARG;
  snprintf(buf, n, "%s", g_last_error.c_str());
  return 0;
}

int cube_gpu_create(const cube_params* p, int device, cube_ctx** out) {
  if (!p || !out) return fail(CUBE_E_ARG, "null argument");
  *out = nullptr;
  if (p->ratio_cs <= 0 || p->ng % p->ratio_cs || (p->ng / p->ratio_cs) % p->nnt ||
      ((p->ng / p->ratio_cs) / p->nnt) % p->nns)
    return fail(CUBE_E_ARG, "ng, nnt, nns must divide evenly (parameters.f90:57-59)");
  if (p->izipx != 1 && p->izipx != 2) return fail(CUBE_E_ARG, "izipx must be 1 or 2");
  if (p->mass_p_cdm <= 0.f) return fail(CUBE_E_ARG, "mass_p_cdm must be positive");
  if (p->nslab < 0 || (p->nslab > 1 && (p->nnt % p->nslab || p->slab < 0 || p->slab >= p->nslab)))
    return fail(CUBE_E_ARG, "nslab must divide nnt, and 0 <= slab < nslab");
  if ((double)(p->ng / p->ratio_cs) * (p->ng / p->ratio_cs) * (p->ng / p->ratio_cs) >= 4294967296.0)
    return fail(CUBE_E_ARG, "at most 2^32 - 1 coarse cells (ng/ratio_cs < 1626)");
  cube_ctx* c = new cube_ctx();
  c->P = *p;
  c->G = make_geo(*p);
  const Geo& G = c->G;
  if (G.nt < 2 * G.ncb) {
    delete c;
    return fail(CUBE_E_ARG, "tiles must be at least 2*ncb coarse cells wide");
  }
  if (G.nt + 2 * G.ncb > 256 || G.ntt < 2) {
    delete c;
    return fail(CUBE_E_ARG, "unsupported tile geometry (nt+2ncb<=256, ntt>=2)");
  }
  c->device = device;
  {
    const char* e = getenv("CUBE_FFT_GENERIC");
    c->fft_generic = (e && e[0] == '1') ? 1 : 0;
    const char* f = getenv("CUBE_FFT_FUSED");
    c->fft_fused = (f && f[0] == '0') ? 0 : 1;
  }
  c->ns3 = (int)((int64_t)G.nnt * G.nnt * G.nnt * G.nns * G.nns * G.nns);
  c->ntiles = G.nnt * G.nnt * G.nnt;
  c->xbytes = G.izipx;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
  CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
  for (int i = 0; i < 8; ++i) CK(cudaEventCreate(&c->ev[i]));
  int rc = add_fft(c, G.nc);
  if (!rc) rc = add_fft(c, G.ngt);
  for (int i = 2; i <= 5 && !rc; ++i) rc = add_fft(c, G.nft[i]);
  if (rc) {
    cube_gpu_destroy(c);
    return rc;
  }
  const size_t big = 200 * 1024;
  CK(cudaFuncSetAttribute(k_fft_x_r2c<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  CK(cudaFuncSetAttribute(k_fft_x_r2c<long long>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  CK(cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  CK(cudaFuncSetAttribute(k_fft_z_green, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  CK(cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  CK(cudaFuncSetAttribute(k_drift_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
  // cells
  const int64_t nc3 = G.ncells;
  CK(cudaMalloc(&c->rhoc, nc3 * 4));
  CK(cudaMalloc(&c->rhoc2, nc3 * 4));
  CK(cudaMalloc(&c->fill, nc3 * 4));
  CK(cudaMalloc(&c->biglist, nc3 * 4));
  CK(cudaMalloc(&c->hugelist, nc3 * 4));
  CK(cudaMalloc(&c->nbig, 8));
  CK(cudaMalloc(&c->cstart, (nc3 + 1) * 8));
  CK(cudaMalloc(&c->cstart2, (nc3 + 1) * 8));
  CK(cudaMalloc(&c->scan_tmp, ((nc3 + 2047) / 2048 + 2) * 8));
  CK(cudaMalloc(&c->rdev, sizeof(StepRes)));
  CK(cudaMemset(c->rdev, 0, sizeof(StepRes)));
  CK(cudaMallocHost(&c->rhost, sizeof(StepRes)));
  c->red = c->rdev->red;
  c->pairs = &c->rdev->pairs;
  c->msum = c->rdev->msum;
  c->mom = c->rdev->mom;
  c->err = &c->rdev->err;
  c->overflow = &c->rdev->overflow;
  c->napm = c->rdev->napm;
  c->total = &c->rdev->total;
  CK(cudaMalloc(&c->sd, sizeof(StepDev)));
  CK(cudaMemset(c->sd, 0, sizeof(StepDev)));
  CK(cudaMallocHost(&c->h_sd, sizeof(StepDev)));
  CK(cudaMalloc(&c->ires, c->ns3 * 4));
  CK(cudaMallocHost(&c->h_ires, c->ns3 * 4));
  if (G.nslab > 1) {  // layer exchange: counts and prefixes of the four layers
    const int64_t nlay = (int64_t)G.nnt * G.nnt * G.ncb * G.nt * G.nt;
    CK(cudaMalloc(&c->lay_cnt, 4 * nlay * 4));
    CK(cudaMalloc(&c->lay_start, 4 * (nlay + 1) * 8));
  }
  if (c->P.pp_queue) {
    if (!(G.izipx == 1 || G.nt < 127)) {
      cube_gpu_destroy(c);
      return fail(CUBE_E_ARG, "pp_queue needs int8 codes, or int16 with nt < 127 (exact FP32 candidates)");
    }
    CK(cudaMalloc(&c->hlist, nc3 * 4));
    CK(cudaMalloc(&c->hpre, (nc3 + 1) * 4));
    CK(cudaMalloc(&c->ppq, PPQ_Q * 4));
    CK(cudaMalloc(&c->tune_red, 32 * 4));
  }
  // Green tables of PM1 and PM2 (initialize.f90:247-258); PM3 classes on first use.
  rc = build_green(c, &c->green1, G.nc, G.apm1c, 0.f, (float)G.rcs);
  if (!rc) rc = build_green(c, &c->green2, G.ngt, G.apm2, G.apm1c * (float)G.rcs, 1.f);
  if (rc) {
    cube_gpu_destroy(c);
    return rc;
  }
  CK(cudaStreamSynchronize(c->s));
  *out = c;
  return 0;
}

int cube_gpu_destroy(cube_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->ck_thread.joinable()) c->ck_thread.join();
  if (c->s3) cudaStreamSynchronize(c->s3);
  if (c->s) cudaStreamSynchronize(c->s);
  drop_graphs(c);
  void* bufs[] = {c->xp, c->xp2, c->vp, c->vp2, c->pid, c->pid2, c->pcell, c->pcell2, c->rhoc, c->rhoc2,
                  c->fill, c->biglist, c->hugelist, c->nbig, c->cstart, c->cstart2, c->scan_tmp, c->dest, c->key, c->skey,
                  c->ssrc, c->rdev, c->sd, c->ires, c->box_slot, c->box_sub, c->arena, c->green1, c->green2,
                  c->cap_buf, c->pfin, c->hperm, c->hlist, c->hpre, c->ppq, c->vtune, c->tune_red, c->tf1, c->tf2,
                  c->nu_tab, c->lay_cnt, c->lay_start, c->lay_buf};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (int i = 0; i < 8; ++i) {
    if (c->green3[i]) cudaFree(c->green3[i]);
    if (c->tf3[i]) cudaFree(c->tf3[i]);
  }
  for (auto& t : c->ffts) cudaFree(t.tw);
  if (c->rhost) cudaFreeHost(c->rhost);
  if (c->ck_host) cudaFreeHost(c->ck_host);
  if (c->ev_ckpt) cudaEventDestroy(c->ev_ckpt);
  if (c->s3) cudaStreamDestroy(c->s3);
  if (c->h_sd) cudaFreeHost(c->h_sd);
  if (c->h_ires) cudaFreeHost(c->h_ires);
  for (int i = 0; i < 8; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
  if (c->s2) cudaStreamSynchronize(c->s2);
  if (c->ev_up) cudaEventDestroy(c->ev_up);
  if (c->ev_drift) cudaEventDestroy(c->ev_drift);
  if (c->s2) cudaStreamDestroy(c->s2);
  if (c->s) cudaStreamDestroy(c->s);
  delete c;
  return 0;
}

// Work on the context stream that overwrites the particle buffers of a checkpoint still
// being copied waits for those copies (a no-op once they are done).  Not inside a
// capture: a replayed step graph waits before its launch instead.
static void after_checkpoint_copy(cube_ctx* c) {
  if (c->ckpt_pending && !c->cap_graph) cudaStreamWaitEvent(c->s, c->ev_ckpt, 0);
}

static int alloc_particles(cube_ctx* c, int64_t np) {
  if (np <= c->cap) return 0;
  drop_graphs(c);
  if (c->ckpt_pending) cudaEventSynchronize(c->ev_ckpt);  // its copies read the buffers freed here
  int64_t cap = std::max<int64_t>(np, c->P.np_capacity);
  if (c->G.nslab > 1) {  // room for the two ghost layers: 2 ncb of the slab's L*nt cell layers, with margin
    const Geo& g = c->G;
    const double frac = 2.0 * g.ncb / ((double)(g.nnt / g.nslab) * g.nt);
    cap = (int64_t)((double)cap * (1.0 + 1.5 * frac)) + 4096;
  }
  void** ps[] = {&c->xp, &c->xp2, (void**)&c->vp, (void**)&c->vp2, (void**)&c->pid, (void**)&c->pid2,
                 (void**)&c->pcell, (void**)&c->pcell2, (void**)&c->dest, (void**)&c->key, (void**)&c->skey,
                 (void**)&c->ssrc};
  const size_t sz[] = {(size_t)cap * 3 * c->xbytes, (size_t)cap * 3 * c->xbytes, (size_t)cap * 12, (size_t)cap * 12,
                       (size_t)cap * 8, (size_t)cap * 8, (size_t)cap * 4, (size_t)cap * 4, (size_t)cap * 4,
                       (size_t)cap * 8, (size_t)cap * 8, (size_t)cap * 4};
  for (int i = 0; i < 12; ++i) {
    if (*ps[i]) cudaFree(*ps[i]);
    *ps[i] = nullptr;
    CK(cudaMalloc(ps[i], sz[i] + 16));
  }
  c->cap = cap;
  c->xp_base = c->xp;
  if (c->P.pp_queue) {
    if (c->pfin) cudaFree(c->pfin);
    if (c->vtune) cudaFree(c->vtune);
    if (c->hperm) cudaFree(c->hperm);
    c->pfin = nullptr;
    c->vtune = nullptr;
    c->hperm = nullptr;
    CK(cudaMalloc(&c->pfin, (size_t)cap * sizeof(float4)));
    CK(cudaMalloc(&c->hperm, (size_t)cap * sizeof(int32_t)));
  }
  // mesh arena: everything that fits of what the largest level needs, within 70% of free memory
  const Geo& G = c->G;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  size_t need = std::max(mesh_bytes(c, G.nc, 1, fixed), mesh_bytes(c, G.ngt, c->ntiles, fixed));
  need = std::max(need, mesh_bytes(c, G.nft[2], c->ns3, fixed));  // every subtile in the lightest class
  for (int i = 3; i <= 5; ++i)
    need = std::max(need, mesh_bytes(c, G.nft[i], std::max<int64_t>(1, c->ns3 / 16), fixed));
  size_t fre = 0, tot = 0;
  CK(cudaMemGetInfo(&fre, &tot));
  size_t budget = (size_t)(0.7 * (double)fre);
  size_t want = std::min(need, budget);
  want = std::max(want, std::max(mesh_bytes(c, G.nc, 1, fixed), mesh_bytes(c, G.nft[5], 1, fixed)));
  if (c->arena) cudaFree(c->arena);
  c->arena = nullptr;
  CK(cudaMalloc(&c->arena, want));
  c->arena_bytes = want;
  const char* verbose = getenv("CUBE_VERBOSE");
  if (verbose && verbose[0] == '1')
    fprintf(stderr, "cube_gpu: free %.2f GB, mesh budget %.2f GB, arena %.2f GB (largest level wants %.2f GB)\n",
            fre / 1e9, budget / 1e9, want / 1e9, need / 1e9);
  return 0;
}

// Grow the particle buffers to hold `need` particles, keeping the current state (the first
// buffer set, c->np particles); the second set and the per-particle scratch come back
// empty at the new size.
static int grow_particles(cube_ctx* c, int64_t need) {
  if (need <= c->cap) return 0;
  if (c->P.pp_queue && need > INT32_MAX)  // the heavy-cell index array holds 32-bit indices
    return fail(CUBE_E_CAPACITY, "pp_queue indexes particles in 32 bits: at most 2^31 - 1 per context");
  drop_graphs(c);
  if (c->ckpt_pending) cudaEventSynchronize(c->ev_ckpt);
  CK(cudaStreamSynchronize(c->s));
  const int64_t cap = need + need / 4 + 4096;
  void** keep[] = {&c->xp, (void**)&c->vp, (void**)&c->pid, (void**)&c->pcell};
  const size_t kper[] = {(size_t)3 * c->xbytes, 12, 8, 4};
  for (int i = 0; i < 4; ++i) {
    void* nb = nullptr;
    CK(cudaMalloc(&nb, (size_t)cap * kper[i] + 16));
    CK(cudaMemcpy(nb, *keep[i], (size_t)c->np * kper[i], cudaMemcpyDeviceToDevice));
    cudaFree(*keep[i]);
    *keep[i] = nb;
  }
  void** fresh[] = {&c->xp2, (void**)&c->vp2, (void**)&c->pid2, (void**)&c->pcell2, (void**)&c->dest,
                    (void**)&c->key, (void**)&c->skey, (void**)&c->ssrc};
  const size_t fper[] = {(size_t)3 * c->xbytes, 12, 8, 4, 4, 8, 8, 4};
  for (int i = 0; i < 8; ++i) {
    if (*fresh[i]) cudaFree(*fresh[i]);
    *fresh[i] = nullptr;
    CK(cudaMalloc(fresh[i], (size_t)cap * fper[i] + 16));
  }
  if (c->pfin) {
    cudaFree(c->pfin);
    c->pfin = nullptr;
    CK(cudaMalloc(&c->pfin, (size_t)cap * sizeof(float4)));
  }
  if (c->vtune) cudaFree(c->vtune);
  c->vtune = nullptr;  // reallocated by the PP tuner when it next runs
  c->cap = cap;
  c->xp_base = c->xp;
  return 0;
}

int cube_gpu_upload(cube_ctx* c, const void* xp, const float* vp, const int64_t* pid, const int32_t* rhoc,
                    int64_t nplocal) {
  if (!c || !xp || !vp || !pid || !rhoc || nplocal <= 0) return fail(CUBE_E_ARG, "bad upload arguments");
  CK(cudaSetDevice(c->device));
  const Geo& G = c->G;
  int64_t sum = 0;
  for (int64_t i = 0; i < G.ncells; ++i) {
    if (rhoc[i] < 0) return fail(CUBE_E_ARG, "negative rhoc");
    if (rhoc[i] && !owned_cell(G, i)) return fail(CUBE_E_ARG, "rhoc holds particles outside this rank's slab");
    sum += rhoc[i];
  }
  if (sum != nplocal) return fail(CUBE_E_COUNT, "sum(rhoc) != nplocal");
  int rc = alloc_particles(c, nplocal);
  if (rc) return rc;
  c->np = nplocal;
  c->own0 = 0;
  c->own1 = nplocal;
  c->ghosts = false;
  after_checkpoint_copy(c);
  CK(cudaMemcpyAsync(c->xp, xp, (size_t)nplocal * 3 * c->xbytes, cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->vp, vp, (size_t)nplocal * 12, cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->pid, pid, (size_t)nplocal * 8, cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->rhoc, rhoc, (size_t)G.ncells * 4, cudaMemcpyHostToDevice, c->s));
  LAUNCH(c, K_SCAN, 3, exclusive_scan(c->rhoc, c->cstart, G.ncells, c->scan_tmp, c->s));
  LAUNCH(c, K_FILL, 1, k_fill_pcell<<<nblk(G.ncells), 256, 0, c->s>>>(c->cstart, G.ncells, c->pcell));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->s));
  c->loaded = true;
  c->have_est = false;
  c->maxcount_est = -1;
  return 0;
}

int cube_gpu_download(cube_ctx* c, void* xp, float* vp, int64_t* pid, int32_t* rhoc, int64_t* nplocal) {
  if (!c || !c->loaded) return fail(CUBE_E_STATE, "no particles on device");
  CK(cudaSetDevice(c->device));
  // this rank's particles: all of them with one slab; the store may also hold ghosts
  const bool slabs = c->G.nslab > 1;
  const int64_t o = slabs ? c->own0 : 0, n = slabs ? c->own1 - c->own0 : c->np;
  if (xp) CK(cudaMemcpyAsync(xp, (char*)c->xp + o * 3 * c->xbytes, (size_t)n * 3 * c->xbytes, cudaMemcpyDeviceToHost, c->s));
  if (vp) CK(cudaMemcpyAsync(vp, c->vp + 3 * o, (size_t)n * 12, cudaMemcpyDeviceToHost, c->s));
  if (pid) CK(cudaMemcpyAsync(pid, c->pid + o, (size_t)n * 8, cudaMemcpyDeviceToHost, c->s));
  if (rhoc) CK(cudaMemcpyAsync(rhoc, c->rhoc, (size_t)c->G.ncells * 4, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  if (rhoc && slabs) {  // ghost cells are other ranks' particles
    memset(rhoc, 0, (size_t)c->G.c0 * 4);
    memset(rhoc + c->G.c1, 0, (size_t)(c->G.ncells - c->G.c1) * 4);
  }
  if (nplocal) *nplocal = n;
  return 0;
}

int64_t cube_gpu_nplocal(cube_ctx* c) {
  if (!c) return fail(CUBE_E_ARG, "null context");
  if (!c->loaded) return 0;
  return c->G.nslab > 1 ? c->own1 - c->own0 : c->np;
}

// Map a device error word to the reference's fatal conditions.
static int err_code(unsigned e) {
  if (e & CUBE_DEVERR_DRIFT_RANGE) return fail(CUBE_E_RANGE, "drift: particle moved beyond the ghost depth");
  if (e & CUBE_DEVERR_SEGMENT) return fail(CUBE_E_CAPACITY, "drift: destination cell exceeds max_segment");
  if (e & CUBE_DEVERR_DEPOSIT_RANGE) return fail(CUBE_E_RANGE, "mass assignment out of range");
  if (e & CUBE_DEVERR_INTERP_RANGE) return fail(CUBE_E_RANGE, "update velocity out of range");
  return fail(CUBE_E_RANGE, "device error word " + std::to_string(e));
}

// Read and clear the device error word (synchronises the stream).
static int check_err(cube_ctx* c) {
  unsigned e = 0;
  CK(cudaMemcpyAsync(&e, c->err, 4, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  if (e) {
    CK(cudaMemsetAsync(c->err, 0, 4, c->s));
    CK(cudaStreamSynchronize(c->s));
    return err_code(e);
  }
  return 0;
}

// The step scalars as the reference derives them (drift.f90:21,26; kick.f90:283-285),
// written to the pinned staging copy; `drift` validates nlayer for a drift.
static int make_scalars(cube_ctx* c, const cube_step_in* in, bool drift, StepDev& d) {
  const Geo& G = c->G;
  d.dt = in->dt;
  d.dt_old = in->dt_old;
  d.a_mid = in->a_mid;
  d.vz_max = in->vz_max;
  d.dt_mid = (in->dt_old + in->dt) / 2.f;
  d.nlayer = 2 * (int)std::ceil(d.dt_mid * in->vz_max / (float)G.rcs) + 2;
  if (drift && (d.nlayer <= 0 || d.nlayer > 65535)) return fail(CUBE_E_ARG, "bad nlayer from dt_mid*vz_max");
  d.pp_mass = (G.f_nu > 0.f) ? (float)((double)G.mass_p * ((1.0 - (double)G.f_nu) * (1.0 - (double)G.f_nu))) : G.mass_p;
  d.pp_vscale = (float)((double)(in->a_mid * in->dt / 6.f) / M_PI);
  return 0;
}

// Stage the scalars and copy them to the device on the context stream (the previous
// step's copy has completed: every step ends with a stream synchronisation).
static int upload_scalars(cube_ctx* c, const StepDev& d) {
  *c->h_sd = d;
  CK(cudaMemcpyAsync(c->sd, c->h_sd, sizeof(StepDev), cudaMemcpyHostToDevice, c->s));
  return 0;
}

// Segments beyond the shared-memory sorter: ranked into the scratch arrays c->key (free
// after the scatter) and c->pcell2 (written only by the gather that follows), then copied
// back.  Both kernels exit at once when no segment is listed.
static void enqueue_huge_sort(cube_ctx* c) {
  uint32_t* tsrc = reinterpret_cast<uint32_t*>(c->pcell2);
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_rank_huge<<<(unsigned)c->nsm, HUGE_T, 0, c->s>>>(
                                 c->hugelist, c->nbig + 1, c->rhoc2, c->cstart2, c->skey, c->ssrc, c->key, tsrc));
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_copy_huge<<<(unsigned)c->nsm, 256, 0, c->s>>>(
                                 c->hugelist, c->nbig + 1, c->rhoc2, c->cstart2, c->key, tsrc, c->skey, c->ssrc));
}

// drift.f90, enqueued without any host synchronisation; the drifted arrays land in the
// second buffers and the particle total in StepRes.total.  With `defer_ids` the gather
// leaves the particle ids alone (the new id array is not written): the caller applies the
// drift's permutation (c->ssrc) to them later with k_permute_ids, from c->pid (the ids
// before the drift, c->pid2 after swap_drift) into c->pid2 (c->pid after it).
static void enqueue_drift(cube_ctx* c, bool defer_ids) {
  const Geo& G = c->G;
  const int64_t np = c->np;
  after_checkpoint_copy(c);
  cudaMemsetAsync(c->rhoc2, 0, G.ncells * 4, c->s);
  cudaMemsetAsync(c->fill, 0, G.ncells * 4, c->s);
  cudaMemsetAsync(c->nbig, 0, 8, c->s);
  LAUNCH(c, K_DRIFT_DEST, 1, k_drift_dest<<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->vp, c->pcell, c->cstart, c->sd,
                                                                     c->dest, c->key, c->rhoc2, c->err));
  LAUNCH(c, K_SCAN, 3, exclusive_scan(c->rhoc2, c->cstart2, G.ncells, c->scan_tmp, c->s));
  LAUNCH(c, K_DRIFT_SCATTER, 1, k_drift_scatter<<<nblk(np), 256, 0, c->s>>>(np, c->dest, c->key, c->cstart2, c->fill, c->skey, c->ssrc));
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_sort_small<<<nblk((G.ncells + 1) / 2 * 32), 256, 0, c->s>>>(G.ncells, c->rhoc2, c->cstart2, c->skey, c->ssrc,
                                                            c->biglist, c->nbig));
  // long segments: one block per SM, each looping over the listed cells
  const int max_seg = c->P.max_segment > 0 ? std::min(c->P.max_segment, 16384) : 16384;
  const unsigned nbb = (unsigned)std::min<int64_t>(G.ncells, c->nsm);
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_sort_big<<<nbb, 512, drift_sort_smem(max_seg), c->s>>>(c->biglist, c->nbig, c->rhoc2, c->cstart2, c->skey,
                                                                   c->ssrc, max_seg, c->hugelist, c->nbig + 1));
  enqueue_huge_sort(c);
  LAUNCH(c, K_DRIFT_GATHER, 1, k_drift_gather<<<nblk(np), 256, 0, c->s>>>(G, np, c->ssrc, c->dest, c->xp, c->vp,
                                                                        defer_ids ? nullptr : c->pid, c->sd, c->xp2, c->vp2,
                                                                        c->pid2, c->pcell2, c->cstart2 + G.ncells));
  cudaMemcpyAsync(c->total, c->cstart2 + G.ncells, 8, cudaMemcpyDeviceToDevice, c->s);
}

// The drift's outputs become the current particle state (host pointers only).
static void swap_drift(cube_ctx* c) {
  std::swap(c->xp, c->xp2);
  std::swap(c->vp, c->vp2);
  std::swap(c->pid, c->pid2);
  std::swap(c->pcell, c->pcell2);
  std::swap(c->rhoc, c->rhoc2);
  std::swap(c->cstart, c->cstart2);
}

// ---- runs split into z-slabs (cube_params.nslab > 1) ----
static int comm_allreduce(cube_ctx* c, void* buf, int64_t count, int dtype, int op, int device) {
  if (!c->have_comm || !c->comm.allreduce) return fail(CUBE_E_STATE, "nslab > 1 needs cube_gpu_set_comm first");
  if (device) CK(cudaStreamSynchronize(c->s));
  const int r = c->comm.allreduce(c->comm.user, buf, count, dtype, op, device);
  if (r) return fail(CUBE_E_COMM, "cube_comm allreduce returned " + std::to_string(r));
  return 0;
}

static int comm_sendrecv(cube_ctx* c, const void* up, int64_t sn_up, const void* down, int64_t sn_down, void* below,
                         int64_t rn_below, void* above, int64_t rn_above, int device) {
  if (!c->have_comm || !c->comm.sendrecv) return fail(CUBE_E_STATE, "nslab > 1 needs cube_gpu_set_comm first");
  if (device) CK(cudaStreamSynchronize(c->s));
  const int r = c->comm.sendrecv(c->comm.user, up, sn_up, down, sn_down, below, rn_below, above, rn_above, device);
  if (r) return fail(CUBE_E_COMM, "cube_comm sendrecv returned " + std::to_string(r));
  return 0;
}

// The four ghost-exchange layers of this slab: 0 the layer it sends down (its lowest ncb
// cell layers), 1 the layer it sends up (its highest), 2 its ghosts from below (the slab
// below's highest layers), 3 its ghosts from above (the slab above's lowest).
static void slab_layer(const Geo& G, int k, int& tz, int& lz0) {
  const int L = G.nnt / G.nslab, tlo = G.tile0 / (G.nnt * G.nnt), thi = tlo + L - 1;
  if (k == 0) {
    tz = tlo;
    lz0 = 0;
  } else if (k == 1) {
    tz = thi;
    lz0 = G.nt - G.ncb;
  } else if (k == 2) {
    tz = (tlo - 1 + G.nnt) % G.nnt;
    lz0 = G.nt - G.ncb;
  } else {
    tz = (thi + 1) % G.nnt;
    lz0 = 0;
  }
}

// Rebuild the store as this rank's particles plus fresh ghost layers from both neighbours
// (the buffer_x/buffer_v step of main.f90:36-38); ghosts of an earlier exchange are
// dropped.  The store keeps the global storage order over the slab's cells and both
// layers, so every kernel reads a ghost cell like any other.  Host synchronisations: the
// layer sizes and the new cell starts are read back.
static int slab_exchange(cube_ctx* c) {
  const Geo& G = c->G;
  const int64_t nlay = (int64_t)G.nnt * G.nnt * G.ncb * G.nt * G.nt;
  int32_t* cnt[4];
  int64_t* st[4];
  int tz[4], lz[4];
  for (int k = 0; k < 4; ++k) {
    cnt[k] = c->lay_cnt + k * nlay;
    st[k] = c->lay_start + k * (nlay + 1);
    slab_layer(G, k, tz[k], lz[k]);
  }
  after_checkpoint_copy(c);
  for (int k = 0; k < 2; ++k) {  // outgoing counts and their prefixes
    LAUNCH(c, K_SLAB, 1, k_layer_counts<<<nblk(nlay), 256, 0, c->s>>>(G, tz[k], lz[k], nlay, c->rhoc, cnt[k]));
    LAUNCH(c, K_SLAB, 3, exclusive_scan(cnt[k], st[k], nlay, c->scan_tmp, c->s));
  }
  int64_t nout[2] = {0, 0}, nin[2] = {0, 0}, own[2] = {0, 0};
  CK(cudaMemcpyAsync(&nout[0], st[0] + nlay, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(&nout[1], st[1] + nlay, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(&own[0], c->cstart + G.c0, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(&own[1], c->cstart + G.c1, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  // sizes, counts, then the particles
  int rc = comm_sendrecv(c, &nout[1], 8, &nout[0], 8, &nin[0], 8, &nin[1], 8, 0);
  if (!rc) rc = comm_sendrecv(c, cnt[1], nlay * 4, cnt[0], nlay * 4, cnt[2], nlay * 4, cnt[3], nlay * 4, 1);
  if (rc) return rc;
  const LayerBuf lb[4] = {layer_buf(nout[0], c->xbytes), layer_buf(nout[1], c->xbytes), layer_buf(nin[0], c->xbytes),
                          layer_buf(nin[1], c->xbytes)};
  size_t off[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < 4; ++k) off[k + 1] = off[k] + (((size_t)lb[k].bytes + 255) & ~(size_t)255);
  if (off[4] > c->lay_bytes) {
    if (c->lay_buf) cudaFree(c->lay_buf);
    c->lay_buf = nullptr;
    c->lay_bytes = 0;
    const size_t want = off[4] + off[4] / 4 + 4096;
    CK(cudaMalloc(&c->lay_buf, want));
    c->lay_bytes = want;
  }
  for (int k = 0; k < 2; ++k)
    LAUNCH(c, K_SLAB, 1, k_layer_pack<<<nblk(nlay), 256, 0, c->s>>>(G, tz[k], lz[k], nlay, c->cstart, st[k], c->xp, c->vp,
                                                                     c->pid, c->lay_buf + off[k], nout[k]));
  rc = comm_sendrecv(c, c->lay_buf + off[1], lb[1].bytes, c->lay_buf + off[0], lb[0].bytes, c->lay_buf + off[2],
                     lb[2].bytes, c->lay_buf + off[3], lb[3].bytes, 1);
  if (rc) return rc;
  // the new cell counts: the slab's own, then both ghost layers
  CK(cudaMemsetAsync(c->rhoc2, 0, G.ncells * 4, c->s));
  CK(cudaMemcpyAsync(c->rhoc2 + G.c0, c->rhoc + G.c0, (size_t)(G.c1 - G.c0) * 4, cudaMemcpyDeviceToDevice, c->s));
  for (int k = 2; k < 4; ++k) {
    LAUNCH(c, K_SLAB, 3, exclusive_scan(cnt[k], st[k], nlay, c->scan_tmp, c->s));
    LAUNCH(c, K_SLAB, 1, k_layer_set_counts<<<nblk(nlay), 256, 0, c->s>>>(G, tz[k], lz[k], nlay, cnt[k], c->rhoc2));
  }
  LAUNCH(c, K_SCAN, 3, exclusive_scan(c->rhoc2, c->cstart2, G.ncells, c->scan_tmp, c->s));
  int64_t total = 0, own0 = 0;
  CK(cudaMemcpyAsync(&total, c->cstart2 + G.ncells, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(&own0, c->cstart2 + G.c0, 8, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  const int64_t nown = own[1] - own[0];
  if (total != nown + nin[0] + nin[1]) return fail(CUBE_E_COUNT, "slab exchange: received counts and particles disagree");
  rc = grow_particles(c, total);
  if (rc) return rc;
  // this rank's particles move as one block; the ghosts go to their cells' starts
  CK(cudaMemcpyAsync((char*)c->xp2 + own0 * 3 * c->xbytes, (char*)c->xp + own[0] * 3 * c->xbytes,
                     (size_t)nown * 3 * c->xbytes, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(c->vp2 + 3 * own0, c->vp + 3 * own[0], (size_t)nown * 12, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(c->pid2 + own0, c->pid + own[0], (size_t)nown * 8, cudaMemcpyDeviceToDevice, c->s));
  for (int k = 2; k < 4; ++k)
    LAUNCH(c, K_SLAB, 1, k_layer_unpack<<<nblk(nlay), 256, 0, c->s>>>(G, tz[k], lz[k], nlay, c->cstart2, st[k],
                                                                       c->lay_buf + off[k], nin[k - 2], c->xp2, c->vp2,
                                                                       c->pid2));
  LAUNCH(c, K_FILL, 1, k_fill_pcell<<<nblk(G.ncells), 256, 0, c->s>>>(c->cstart2, G.ncells, c->pcell2));
  CK(cudaGetLastError());
  std::swap(c->xp, c->xp2);
  std::swap(c->vp, c->vp2);
  std::swap(c->pid, c->pid2);
  std::swap(c->pcell, c->pcell2);
  std::swap(c->rhoc, c->rhoc2);
  std::swap(c->cstart, c->cstart2);
  c->np = total;
  c->own0 = own0;
  c->own1 = own0 + nown;
  c->ghosts = true;
  return 0;
}

// After a drift of a split run: the store holds only the particles that landed in this
// slab; the total over the slabs must not change (drift.f90:139-143 checks it per image).
static int slab_after_drift(cube_ctx* c, int64_t nown_before, int64_t total) {
  c->np = total;
  c->own0 = 0;
  c->own1 = total;
  c->ghosts = false;
  int64_t n[2] = {nown_before, total};
  const int rc = comm_allreduce(c, n, 2, CUBE_DT_I64, CUBE_OP_SUM, 0);
  if (rc) return rc;
  if (n[0] != n[1]) return fail(CUBE_E_COUNT, "drift: particle count not conserved over the slabs");
  return 0;
}

int cube_gpu_drift(cube_ctx* c, const cube_step_in* in) {
  if (!c || !in) return fail(CUBE_E_ARG, "null argument");
  if (!c->loaded) return fail(CUBE_E_STATE, "drift before upload");
  CK(cudaSetDevice(c->device));
  StepDev d;
  int rc = make_scalars(c, in, true, d);
  if (!rc) rc = upload_scalars(c, d);
  if (!rc && c->G.nslab > 1 && !c->ghosts) rc = slab_exchange(c);
  if (rc) return rc;
  const int64_t nown = c->own1 - c->own0;
  enqueue_drift(c, false);
  CK(cudaGetLastError());
  swap_drift(c);
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, c->total, 8, cudaMemcpyDeviceToHost, c->s));
  rc = check_err(c);
  prof_collect(c);
  if (rc) return rc;
  if (c->G.nslab > 1) return slab_after_drift(c, nown, total);
  if (total != c->np) return fail(CUBE_E_COUNT, "drift: particle count not conserved");
  return 0;
}

static float dt_crit(float coef, float f2max, float a_mid) {
  const float G_grid = (float)((double)(1.0f / 6.0f) / M_PI);  // variables.f90:28
  return coef * std::sqrt(1.f / (std::sqrt(f2max) * a_mid * G_grid));
}

// ---- the kick in stages ----
// PM1 and PM2, then the subtile classes.  Zeroes the kick's reductions first.
static int enqueue_kick_a(cube_ctx* c) {
  const Geo& G = c->G;
  const int64_t np = c->np;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  float* f2 = c->red;        // [0..3]
  float* vm = c->red + 8;    // [pm2 0..2][pm3 3..5][pp 6..8]
  CK(cudaMemsetAsync(c->red, 0, 64 * sizeof(float), c->s));
  CK(cudaMemsetAsync(c->pairs, 0, 16, c->s));
  CK(cudaMemsetAsync(c->msum, 0, 3 * MASS_SLOTS * MASS_STRIDE * 8, c->s));
  unsigned long long* ms1 = c->msum;
  unsigned long long* ms2 = c->msum + MASS_SLOTS * MASS_STRIDE;
  CK(mark(c, c->ev[0]));
  // ---------------- PM1 (particle_mesh.f90) ----------------
  {
    // this rank's particles: all of them with one slab; a split run sums the density of
    // every rank's particles over the whole box (exact in the fixed-point form) and solves
    // PM1 on each rank
    const int64_t o = G.nslab > 1 ? c->own0 : 0, npo = G.nslab > 1 ? c->own1 - c->own0 : np;
    const void* xpo = static_cast<const char*>(c->xp) + o * 3 * c->xbytes;
    const int32_t* pco = c->pcell + o;
    float* vpo = c->vp + 3 * o;
    const int n = G.nc;
    MeshPtrs m = mesh_ptrs(c, n, 1, fixed);
    CK(cudaMemsetAsync(m.real, 0, mesh_bytes(c, n, 1, fixed), c->s));
    if (fixed)
      LAUNCH(c, K_DEP_PM1, 1, k_deposit_pm1_runs<<<nblk(npo), 256, 0, c->s>>>(G, npo, xpo, pco,
                                                                     reinterpret_cast<unsigned long long*>(m.real), m.pt.pr, m.pt.plr, ms1));
    else LAUNCH(c, K_DEP_PM1, 1, k_deposit_pm1<false><<<nblk(npo), 256, 0, c->s>>>(G, npo, xpo, pco, m.real, m.pt.pr, m.pt.plr, ms1));
    if (G.nslab > 1) {
      const int64_t nel = (int64_t)(mesh_bytes(c, n, 1, fixed) / (fixed ? 8 : 4));
      const int rc = comm_allreduce(c, m.real, nel, fixed ? CUBE_DT_I64 : CUBE_DT_F32, CUBE_OP_SUM, 1);
      if (rc) return rc;
    }
    maybe_capture(c, 1, 0, 0, m.real, n, fixed, m.pt.rp, m.pt.psb);
    float* phi = reinterpret_cast<float*>(m.real);
    const float* k1 = kernel_table(c, 1, 0);
    if (!k1) return CUBE_E_CUDA;
    launch_fft(c, n, 1, m.real, fixed, G.mass_p, phi, m.ck, k1, (float)n, 3, 1);
    maybe_capture(c, 1, 0, 1, phi, n, false, (int64_t)m.pt.pf * 4, m.pt.psb);
    LAUNCH(c, K_F2_PM1, 1, k_f2max_periodic<<<(unsigned)std::min<int64_t>(1184, (int64_t)n * n / 8 + 1), 256, 0, c->s>>>(phi, n, f2 + 0, m.pt.pf, m.pt.plf));
    // force mesh (float4 per coarse cell) in the arena after phi, when it fits
    const size_t foff = (mesh_bytes(c, n, 1, fixed) + 255) & ~(size_t)255;
    const int64_t n3 = (int64_t)n * n * n;
    if (foff + (size_t)n3 * sizeof(float4) <= c->arena_bytes) {
      float4* force = reinterpret_cast<float4*>(reinterpret_cast<char*>(c->arena) + foff);
      LAUNCH(c, K_INT_PM1, 1, k_force_pm1<<<nblk(n3), 256, 0, c->s>>>(n, phi, m.pt.pf, m.pt.plf, force));
      LAUNCH(c, K_INT_PM1, 1, k_interp_pm1_force<<<nblk(npo), 256, 0, c->s>>>(G, npo, xpo, pco, force, vpo, c->sd));
    } else {
      LAUNCH(c, K_INT_PM1, 1, k_interp_pm1<<<nblk(npo), 256, 0, c->s>>>(G, npo, xpo, pco, phi, vpo, c->sd, m.pt.pf, m.pt.plf));
    }
  }
  CK(mark(c, c->ev[1]));
  // ---------------- PM2 (kick.f90:47-77) ----------------
  {
    const int n = G.ngt;
    const int64_t per = std::min<int64_t>(G.tile1 - G.tile0, boxes_fit(c, n, fixed));
    for (int t0 = G.tile0; t0 < G.tile1; t0 += (int)per) {  // this rank's tiles
      const int nb = (int)std::min<int64_t>(per, G.tile1 - t0);
      MeshPtrs m = mesh_ptrs(c, n, nb, fixed);
      const int64_t boxb = (int64_t)n * m.pt.psb;
      CK(cudaMemsetAsync(m.real, 0, nb * boxb, c->s));
      if (fixed) LAUNCH(c, K_DEP_PM2, 1, k_deposit_pm2<true><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, m.real, t0, nb, m.pt.pr, m.pt.plr, ms2));
      else LAUNCH(c, K_DEP_PM2, 1, k_deposit_pm2<false><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, m.real, t0, nb, m.pt.pr, m.pt.plr, ms2));
      if (c->cap_level == 2 && c->cap_box >= t0 && c->cap_box < t0 + nb)
        maybe_capture(c, 2, c->cap_box, 0, (char*)m.real + (c->cap_box - t0) * boxb, n, fixed, m.pt.rp, m.pt.psb);
      float* phi = reinterpret_cast<float*>(m.real);
      const float* k2 = kernel_table(c, 2, 0);
      if (!k2) return CUBE_E_CUDA;
      launch_fft(c, n, nb, m.real, fixed, G.mass_p, phi, m.ck, k2, (float)n * (float)n * (float)n, 1, 2);
      if (c->cap_level == 2 && c->cap_box >= t0 && c->cap_box < t0 + nb)
        maybe_capture(c, 2, c->cap_box, 1, (char*)m.real + (c->cap_box - t0) * boxb, n, false, (int64_t)m.pt.pf * 4,
                      m.pt.psb);
      LAUNCH(c, K_F2_PM2, 1, k_f2max_box2<<<f2max_box2_grid(G.ngp, nb), 256, 0, c->s>>>(phi, n, G.ngp, 1 - G.ngb, nb, f2 + 1, m.pt.pf, m.pt.plf, nullptr));
      LAUNCH(c, K_INT_PM2, 1, k_interp_pm2<<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, phi, t0, nb, c->vp, c->sd, vm + 0, c->err, m.pt.pf, m.pt.plf));
    }
  }
  CK(mark(c, c->ev[2]));
  // ---------------- subtile classes (kick.f90:108-138) ----------------
  CK(cudaMemsetAsync(c->napm, 0, 32, c->s));
  LAUNCH(c, K_CLASSIFY, 1, k_classify<<<nblk(c->ns3), 256, 0, c->s>>>(G, c->rhoc, c->ns3, c->ires, c->napm));
  if (G.nslab > 1) {  // every rank's classes (the PM3 mass needs its neighbours')
    const int rc = comm_allreduce(c, c->ires, c->ns3, CUBE_DT_I32, CUBE_OP_MAX, 1);
    if (rc) return rc;
  }
  if (c->P.pp_queue && c->P.pp_on) {  // the PP tuning class of this step
    CK(cudaMemsetAsync(&c->rdev->maxcount, 0, 4, c->s));
    LAUNCH(c, K_CLASSIFY, 1, k_ppq_maxcount<<<(unsigned)std::min<int64_t>(nblk(G.c1 - G.c0), 4 * c->nsm), 256, 0, c->s>>>(
                                c->cstart, G.c0, G.c1, &c->rdev->maxcount));
  }
  // PM3 mass over the boxes' physical cells, from the classes just found
  if (c->P.pm3_on) {
    unsigned long long* ms3 = c->msum + 2 * MASS_SLOTS * MASS_STRIDE;
    if (fixed) LAUNCH(c, K_MASS, 1, k_mass_pm3<true><<<nblk(G.ncells), 256, 0, c->s>>>(G, c->cstart, c->xp, c->ires, ms3));
    else LAUNCH(c, K_MASS, 1, k_mass_pm3<false><<<nblk(G.ncells), 256, 0, c->s>>>(G, c->cstart, c->xp, c->ires, ms3));
  }
  return 0;
}

// PM3 chunk plan for class counts `cnt`: exact (cap = count) or with headroom for a
// captured step (present classes +1/32, at least 2 boxes; absent classes none: a padded
// slot still costs its FFT).  `skip` (may be null) leaves out the first skip[c] subtiles
// of each class, the ones a captured step already covered.
static PM3Plan make_plan(cube_ctx* c, const int32_t cnt[8], bool headroom, const int* skip = nullptr) {
  const Geo& G = c->G;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  PM3Plan pl;
  memset(&pl, 0, sizeof(pl));
  int k = 0;
  pl.per_max = 1;
  for (int cl = 2; cl <= 5; ++cl) {
    pl.skip[cl] = skip ? skip[cl] : 0;
    int64_t want = std::max<int64_t>(0, (int64_t)cnt[cl] - pl.skip[cl]);
    if (headroom && want > 0) want = want + std::max<int64_t>(2, want / 32);
    want = std::min<int64_t>(want, c->ns3);
    pl.cap[cl] = (int)want;
    if (want == 0 || !c->P.pm3_on) {
      pl.cap[cl] = 0;
      continue;
    }
    const bool lint = fixed && !dep3_own_fits(G, cl);
    const int64_t per = std::min<int64_t>(want, boxes_fit(c, G.nft[cl], lint));
    pl.per[cl] = (int)per;
    pl.kbase[cl] = k;
    k += (int)((want + per - 1) / per);
    pl.per_max = std::max<int>(pl.per_max, (int)per);
  }
  pl.nk = k;
  return pl;
}

// Room for a plan's lists.  Growing them invalidates captured steps (they hold the old
// pointers); the stream has no work that uses them when this runs.
static int ensure_plan_buffers(cube_ctx* c, const PM3Plan& pl) {
  const int64_t ns = std::max<int64_t>(1, (int64_t)pl.nk) * c->ns3;
  const int64_t nsub = std::max<int64_t>(1, (int64_t)pl.nk) * pl.per_max;
  if (ns <= c->slot_cap && nsub <= c->sub_cap) return 0;
  drop_graphs(c);
  if (c->box_slot) cudaFree(c->box_slot);
  if (c->box_sub) cudaFree(c->box_sub);
  c->box_slot = c->box_sub = nullptr;
  c->slot_cap = c->sub_cap = 0;
  CK(cudaMalloc(&c->box_slot, ns * 4));
  CK(cudaMalloc(&c->box_sub, nsub * 4));
  c->slot_cap = ns;
  c->sub_cap = nsub;
  return 0;
}

// The class lists of a plan, built on the device from ires.
static int enqueue_lists(cube_ctx* c, const PM3Plan& pl) {
  if (pl.nk == 0) return 0;
  CK(cudaMemsetAsync(c->box_slot, 0xff, (size_t)pl.nk * c->ns3 * 4, c->s));
  CK(cudaMemsetAsync(c->box_sub, 0xff, (size_t)pl.nk * pl.per_max * 4, c->s));
  LAUNCH(c, K_CLASSIFY, 1, k_build_lists<<<1, 1024, 0, c->s>>>(c->ires, c->ns3, c->G.s0, c->G.s1, pl, c->box_slot,
                                                               c->box_sub, c->overflow));
  return 0;
}

// Slot of subtile s in its chunk of a plan (host copy of ires), for test captures.
static int host_slot(const cube_ctx* c, const PM3Plan& pl, int s, int& chunk) {
  const int cl = c->h_ires[s];
  int rank = -pl.skip[cl];
  for (int t = 0; t < s; ++t) rank += c->h_ires[t] == cl;
  if (rank < 0 || rank >= pl.cap[cl]) return -1;
  chunk = pl.kbase[cl] + rank / pl.per[cl];
  return rank % pl.per[cl];
}

// PM3 (kick.f90:203-276) over the plan's chunks.  Each particle takes its PM3 kick from
// its own subtile's box only, so the boxes can be split over passes.  `host_ires` marks
// that h_ires holds this step's classes (test captures of a PM3 box need it).
static int enqueue_pm3(cube_ctx* c, const PM3Plan& pl, bool host_ires) {
  if (!c->P.pm3_on) return 0;
  const Geo& G = c->G;
  const int64_t np = c->np;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  float* f2 = c->red;
  float* vm = c->red + 8;
  int cap_chunk = -1, cap_slot = -1;
  if (host_ires && c->cap_level == 3 && c->cap_box >= 0 && c->cap_box < c->ns3)
    cap_slot = host_slot(c, pl, c->cap_box, cap_chunk);
  for (int cl = 2; cl <= 5; ++cl) {
    if (pl.cap[cl] == 0) continue;
    const int n = G.nft[cl];
    const float* g3 = kernel_table(c, 3, cl);
    if (!g3) return CUBE_E_CUDA;
    const bool own = fixed && dep3_own_fits(G, cl);
    const bool lint = fixed && !own;  // int64 mesh layout
    const int nch = (pl.cap[cl] + pl.per[cl] - 1) / pl.per[cl];
    for (int ch = 0; ch < nch; ++ch) {
      const int k = pl.kbase[cl] + ch;
      const int nb = std::min(pl.per[cl], pl.cap[cl] - ch * pl.per[cl]);
      const int32_t* slots = c->box_slot + (int64_t)k * c->ns3;
      const int32_t* subs = c->box_sub + (int64_t)k * pl.per_max;
      MeshPtrs m = mesh_ptrs(c, n, nb, lint);
      const int64_t boxb = (int64_t)n * m.pt.psb;
      if (own) {
        // owner-computes deposit: writes every cell (as float), no memset
        const int nr = (n + DEP3_R - 1) / DEP3_R, nrz = (n + DEP3_RZ - 1) / DEP3_RZ;
        const size_t sm = (size_t)DEP3_R * DEP3_R * DEP3_RZ * 8;
        smem_optin(k_deposit_pm3_own, sm);
        LAUNCH(c, K_DEP_PM3, 1, k_deposit_pm3_own<<<(unsigned)((int64_t)nb * nr * nr * nrz), DEP3_THREADS, sm, c->s>>>(
                                    G, c->xp, c->cstart, subs, cl, reinterpret_cast<float*>(m.real), c->err, m.pt.pr,
                                    m.pt.plr, nr, nr, nrz));
      } else {
        CK(cudaMemsetAsync(m.real, 0, nb * boxb, c->s));
        if (fixed) LAUNCH(c, K_DEP_PM3, 1, k_deposit_pm3<true><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, slots, cl, m.real, c->err, m.pt.pr, m.pt.plr));
        else LAUNCH(c, K_DEP_PM3, 1, k_deposit_pm3<false><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, slots, cl, m.real, c->err, m.pt.pr, m.pt.plr));
      }
      const bool cap_here = cap_slot >= 0 && cap_chunk == k;
      if (cap_here) maybe_capture(c, 3, c->cap_box, 0, (char*)m.real + cap_slot * boxb, n, lint, m.pt.rp, m.pt.psb);
      float* phi = reinterpret_cast<float*>(m.real);
      launch_fft(c, n, nb, m.real, lint, G.mass_p, phi, m.ck, g3, (float)n * (float)n * (float)n, 1, 3);
      if (cap_here)
        maybe_capture(c, 3, c->cap_box, 1, (char*)m.real + cap_slot * boxb, n, false, (int64_t)m.pt.pf * 4, m.pt.psb);
      const int nf = G.nfp[cl];
      LAUNCH(c, K_F2_PM3, 1, k_f2max_box2<<<f2max_box2_grid(nf, nb), 256, 0, c->s>>>(phi, n, nf, 1 - G.nfb[cl], nb, f2 + 2, m.pt.pf, m.pt.plf, subs));
      unsigned long long* ms3 = c->msum + 2 * MASS_SLOTS * MASS_STRIDE;
      if (fixed)
        LAUNCH(c, K_INT_PM3, 1, k_interp_pm3<true><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, phi, slots, cl, c->vp,
                                                                               c->sd, vm + 3, c->err, m.pt.pf, m.pt.plf, ms3));
      else
        LAUNCH(c, K_INT_PM3, 1, k_interp_pm3<false><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, phi, slots, cl, c->vp,
                                                                                c->sd, vm + 3, c->err, m.pt.pf, m.pt.plf, ms3));
    }
  }
  return 0;
}

// The queue PP (pp.cuh) with shape sh: offsets, light cells, heavy-cell queue, heavy
// items.  Velocities go from c->vp to vout; f2 (PP f2max), vm (PP vmax[3]) and pairs
// (in range, candidates) receive the reductions.
static void enqueue_ppq(cube_ctx* c, const PPShape& sh, float* vout, float* f2, float* vm, unsigned long long* pairs,
                        const unsigned* abort) {
  const Geo& G = c->G;
  const int64_t np = c->np;
  LAUNCH(c, K_PP, 1, k_ppq_prep<<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pfin));
  LAUNCH(c, K_PP, 1, k_ppq_light<<<nblk(np, PPL_T), PPL_T, 0, c->s>>>(G, np, c->pcell, c->cstart, c->ires, c->pfin,
                                                                      c->vp, vout, c->sd, sh.T, f2, vm, pairs, pairs + 1,
                                                                      abort));
  cudaMemsetAsync(c->ppq, 0, PPQ_Q * 4, c->s);
  LAUNCH(c, K_PP, 1, k_ppq_bucket_count<<<nblk(G.c1 - G.c0), 256, 0, c->s>>>(c->cstart, G.c0, G.c1, sh.T, c->ppq));
  LAUNCH(c, K_PP, 1, k_ppq_bucket_scan<<<1, 32, 0, c->s>>>(c->ppq));
  LAUNCH(c, K_PP, 1, k_ppq_bucket_fill<<<nblk(G.c1 - G.c0), 256, 0, c->s>>>(c->cstart, G.c0, G.c1, sh.T, c->ppq, c->hlist));
  LAUNCH(c, K_PP, 1, k_ppq_items<<<1, 1024, 0, c->s>>>(c->hlist, c->cstart, sh.B, c->ppq, c->hpre));
  LAUNCH(c, K_PP, 1, k_ppq_sort_codes<<<(unsigned)(4 * c->nsm), 256, 0, c->s>>>(G, c->hlist, c->ppq, c->cstart, c->ires,
                                                                                c->pfin, c->hperm));
  const unsigned grid = (unsigned)(c->nsm * std::max(1, 1024 / sh.B));
  const size_t sm = ppq_heavy_smem(sh.B, sh.J);
  smem_optin(k_ppq_heavy, sm);
  LAUNCH(c, K_PP, 1, k_ppq_heavy<<<grid, sh.B, sm, c->s>>>(G, c->hlist, c->hpre, c->ppq, c->cstart, c->ires, c->pfin,
                                                            c->hperm, c->vp, vout, c->sd, sh.J, f2, vm, pairs,
                                                            pairs + 1, abort));
}

// The autotuner of the queue PP: on the current particle state, time every shape of a
// small sweep (light threshold T, item size B, chunk J), writing the velocities to a
// scratch copy, and keep the fastest for occupancy class cls.  Results do not depend on
// the shape (pp.cuh), only the time does.  Runs eagerly (never inside a capture).
static int pp_tune(cube_ctx* c, int cls, int maxcount) {
  if (!c->vtune) CK(cudaMalloc(&c->vtune, (size_t)c->cap * 12));
  const bool prof = c->prof;
  c->prof = false;  // the sweep is not part of any step's kernel profile
  std::vector<PPShape> cands;
  // T descending; B = 512 (one block per SM at the heavy kernel's registers) and J = 1024
  // (the chunk length changes no time measured on 512^3 and 256^3 runs, z = 49 to 0) were
  // never chosen and are left out of the sweep, which runs on the live state; B = 32 (an
  // item of one warp) serves cells of a few dozen particles
  const int Ts[] = {2048, 256, 64, 16}, Bs[] = {32, 128, 256}, Js[] = {256};
  bool all_light_done = false;
  for (int T : Ts) {
    const bool all_light = T >= maxcount;  // no heavy cells: B and J do not matter
    if (all_light && all_light_done) continue;
    all_light_done |= all_light;
    for (int B : Bs)
      for (int J : Js) {
        if (all_light && (B != Bs[2] || J != Js[0])) continue;
        PPShape sh;
        sh.T = T;
        sh.B = B;
        sh.J = J;
        cands.push_back(sh);
      }
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  PPShape win;
  const char* vstr = getenv("CUBE_VERBOSE");
  const bool verbose2 = vstr && vstr[0] == '2';
  for (const PPShape& sh : cands) {
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // the second run is timed
      cudaMemsetAsync(c->tune_red, 0, 32 * 4, c->s);
      cudaEventRecord(e0, c->s);
      enqueue_ppq(c, sh, c->vtune, c->tune_red, c->tune_red + 8,
                  reinterpret_cast<unsigned long long*>(c->tune_red + 16), nullptr);
      cudaEventRecord(e1, c->s);
    }
    const cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      c->prof = prof;
      return fail(CUBE_E_CUDA, std::string("PP tuning: ") + cudaGetErrorString(e));
    }
    cudaEventElapsedTime(&ms, e0, e1);
    if (verbose2) fprintf(stderr, "cube_gpu: PP shape T=%d B=%d J=%d: %.3f ms\n", sh.T, sh.B, sh.J, ms);
    // shapes come with the light threshold T descending; a smaller T (more of the particles
    // in the heavy queue) must win clearly, because cells grow between tunings of a class
    if (ms < best * 0.97f) {
      best = ms;
      win = sh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->prof = prof;
  c->pp_best[cls] = win;
  c->pp_tuned[cls] = true;
  c->pp_tune_ms[cls] = best;
  if (vstr && (vstr[0] == '1' || verbose2))
    fprintf(stderr, "cube_gpu: PP tuned for class %d (max %d per cell): T=%d B=%d J=%d, %.3f ms (%zu shapes)\n", cls,
            maxcount, win.T, win.B, win.J, best, cands.size());
  return 0;
}

// The PP shape for a step whose largest cell holds maxcount particles (tuned on first use).
static int pp_shape(cube_ctx* c, int maxcount, PPShape& sh) {
  const int cls = pp_class(maxcount);
  if (!c->pp_tuned[cls]) {
    const int rc = pp_tune(c, cls, maxcount);
    if (rc) return rc;
  }
  sh = c->pp_best[cls];
  return 0;
}

// PP (kick.f90:280-311), then the FP64 momentum sums of the kicked velocities.  pps:
// the queue PP's shape, or null for one thread per particle (k_pp).
static void enqueue_pp_and_momentum(cube_ctx* c, const unsigned* abort, const PPShape* pps = nullptr) {
  const Geo& G = c->G;
  const int64_t np = c->np;
  float* f2 = c->red;
  float* vm = c->red + 8;
  if (c->P.pp_on && pps) {
    enqueue_ppq(c, *pps, c->vp, f2 + 3, vm + 6, c->pairs, abort);
  } else if (c->P.pp_on) {
    // FP32 candidate positions are exact when lq + offset fits 24 bits: int8 codes, or
    // int16 codes with tile-local coordinates |lq| <= nt < 128
    const bool pp_fast = G.izipx == 1 || G.nt < 127;
    if (pp_fast)
      LAUNCH(c, K_PP, 1, k_pp<true><<<nblk(np, 128), 128, 0, c->s>>>(G, np, c->xp, c->pcell, c->cstart, c->ires, c->vp,
                                                                    c->sd, f2 + 3, vm + 6, c->pairs, c->pairs + 1, abort));
    else
      LAUNCH(c, K_PP, 1, k_pp<false><<<nblk(np, 128), 128, 0, c->s>>>(G, np, c->xp, c->pcell, c->cstart, c->ires, c->vp,
                                                                     c->sd, f2 + 3, vm + 6, c->pairs, c->pairs + 1, abort));
  }
  mark(c, c->ev[4]);
  const int64_t o = G.nslab > 1 ? c->own0 : 0, npo = G.nslab > 1 ? c->own1 - c->own0 : np;
  LAUNCH(c, K_MOMENTUM, 1, k_momentum<<<MOM_BLOCKS, MOM_THREADS, 0, c->s>>>(c->vp + 3 * o, npo, c->mom));
}

// cube_step_out from the step results in c->rhost.
static void fill_out(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  const StepRes& R = *c->rhost;
  const float* red = R.red;
  const float a_mid = in->a_mid;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  memset(out, 0, sizeof(*out));
  out->f2max_pm1 = red[0];
  out->f2max_pm2 = red[1];
  out->f2max_pm3 = red[2];
  out->f2max_pp = red[3];
  out->dt_pm1 = dt_crit(0.5f, red[0], a_mid);  // kick.f90:39
  out->dt_pm2 = dt_crit(0.5f, red[1], a_mid);  // kick.f90:69
  out->dt_pm3 = dt_crit(0.5f, red[2], a_mid);  // kick.f90:239
  out->dt_pp = dt_crit(0.05f, red[3], a_mid);  // kick.f90:298
  const float* v = c->P.pp_on ? (red + 14) : (c->P.pm3_on ? red + 11 : red + 8);
  for (int d = 0; d < 3; ++d) out->vmax[d] = v[d];
  const float vmx = std::max(v[0], std::max(v[1], v[2]));
  out->dt_vmax = 0.9f * 14 / vmx;  // kick.f90:314
  out->vz_max = v[2];
  for (int i = 0; i < 8; ++i) out->napm[i] = R.napm[i];
  out->nplocal = c->G.nslab > 1 ? c->own1 - c->own0 : c->np;
  out->pp_pairs = (int64_t)R.pairs;
  out->pp_candidates = (int64_t)R.cand;
  float ms;
  for (int i = 0; i < 4; ++i) {
    ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]);
    out->tcat[1 + i] = ms;
  }
  ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]);
  out->tcat[5] = ms;
  double mass[3];
  for (int l = 0; l < 3; ++l) {
    const unsigned long long* q = R.msum + l * MASS_SLOTS * MASS_STRIDE;
    if (fixed) {
      unsigned __int128 t = 0;  // exact: 128-bit slots (sum, carries) of int64 contributions
      for (int k = 0; k < MASS_SLOTS; ++k)
        t += ((unsigned __int128)q[k * MASS_STRIDE + 1] << 64) + q[k * MASS_STRIDE];
      mass[l] = std::ldexp((double)(unsigned long long)(t >> 64), 24) + std::ldexp((double)(unsigned long long)t, -40);
    } else {
      double t = 0.0;
      for (int k = 0; k < MASS_SLOTS; ++k) {
        double x;
        memcpy(&x, q + k * MASS_STRIDE, sizeof x);
        t += x;
      }
      mass[l] = t;
    }
  }
  out->mass_pm1 = mass[0];
  out->mass_pm2 = mass[1];
  out->mass_pm3 = mass[2];
  for (int d = 0; d < 3; ++d) {
    double t = 0.0;
    for (int b = 0; b < MOM_BLOCKS; ++b) t += R.mom[3 * b + d];
    out->momentum[d] = t;
  }
}

// The kick (kick.f90:1-353) eagerly: PM1 and PM2, the classes read back, PM3 over exact
// class lists, PP, and the results read back (two host synchronisations).
static int slab_reduce_out(cube_ctx* c, const cube_step_in* in, cube_step_out* out);

static int kick_eager(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  int rc = 0;
  if (c->G.nslab > 1 && !c->ghosts) rc = slab_exchange(c);  // ghosts with this step's positions
  if (!rc) rc = enqueue_kick_a(c);
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->h_ires, c->ires, c->ns3 * 4, cudaMemcpyDeviceToHost, c->s));
  CK(cudaMemcpyAsync(c->rhost->napm, c->napm, 36, cudaMemcpyDeviceToHost, c->s));  // napm and maxcount
  CK(cudaStreamSynchronize(c->s));
  int32_t napm[8];
  memcpy(napm, c->rhost->napm, sizeof napm);
  const PM3Plan pl = make_plan(c, napm, false);
  rc = ensure_plan_buffers(c, pl);
  if (!rc) rc = enqueue_lists(c, pl);
  if (!rc) rc = enqueue_pm3(c, pl, true);
  if (rc) return rc;
  CK(mark(c, c->ev[3]));
  PPShape pps;
  const bool ppq = c->P.pp_queue && c->P.pp_on;
  if (ppq) {
    rc = pp_shape(c, c->rhost->maxcount, pps);
    if (rc) return rc;
  }
  enqueue_pp_and_momentum(c, nullptr, ppq ? &pps : nullptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->rhost, c->rdev, sizeof(StepRes), cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  prof_collect(c);
  memcpy(c->napm_est, c->rhost->napm, sizeof c->napm_est);
  c->have_est = true;
  c->maxcount_est = c->rhost->maxcount;
  if (c->rhost->err) {
    CK(cudaMemsetAsync(c->err, 0, 4, c->s));
    CK(cudaStreamSynchronize(c->s));
    return err_code(c->rhost->err);
  }
  if (c->G.nslab > 1) {
    c->ghosts = false;  // the ghosts' velocities are their owners' business, stale now
    cube_step_out local;
    cube_step_out* o = out ? out : &local;  // every rank takes part in the reductions
    fill_out(c, in, o);
    return slab_reduce_out(c, in, o);
  }
  if (out) fill_out(c, in, out);
  return 0;
}

// The step results over all ranks of a split run (kick.f90:316-346 reduces the dt
// criteria over images): maxima of the f2max and |v| values, sums of the PP pair counts,
// the level masses and the momentum; the dt criteria from the global maxima.
static int slab_reduce_out(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  float mx[8] = {out->f2max_pm1, out->f2max_pm2, out->f2max_pm3, out->f2max_pp, out->vmax[0], out->vmax[1],
                 out->vmax[2], 0.f};
  int64_t si[2] = {out->pp_pairs, out->pp_candidates};
  double sd[6] = {out->mass_pm1, out->mass_pm2, out->mass_pm3, out->momentum[0], out->momentum[1], out->momentum[2]};
  int rc = comm_allreduce(c, mx, 8, CUBE_DT_F32, CUBE_OP_MAX, 0);
  if (!rc) rc = comm_allreduce(c, si, 2, CUBE_DT_I64, CUBE_OP_SUM, 0);
  if (!rc) rc = comm_allreduce(c, sd, 6, CUBE_DT_F64, CUBE_OP_SUM, 0);
  if (rc) return rc;
  const float a_mid = in->a_mid;
  out->f2max_pm1 = mx[0];
  out->f2max_pm2 = mx[1];
  out->f2max_pm3 = mx[2];
  out->f2max_pp = mx[3];
  out->dt_pm1 = dt_crit(0.5f, mx[0], a_mid);
  out->dt_pm2 = dt_crit(0.5f, mx[1], a_mid);
  out->dt_pm3 = dt_crit(0.5f, mx[2], a_mid);
  out->dt_pp = dt_crit(0.05f, mx[3], a_mid);
  for (int d = 0; d < 3; ++d) out->vmax[d] = mx[4 + d];
  out->dt_vmax = 0.9f * 14 / std::max(mx[4], std::max(mx[5], mx[6]));
  out->vz_max = mx[6];
  out->pp_pairs = si[0];
  out->pp_candidates = si[1];
  out->mass_pm1 = sd[0];
  out->mass_pm2 = sd[1];
  out->mass_pm3 = sd[2];
  for (int d = 0; d < 3; ++d) out->momentum[d] = sd[3 + d];
  return 0;
}

int cube_gpu_kick(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  if (!c || !in) return fail(CUBE_E_ARG, "null argument");
  if (!c->loaded) return fail(CUBE_E_STATE, "kick before upload");
  CK(cudaSetDevice(c->device));
  StepDev d;
  int rc = make_scalars(c, in, false, d);
  if (!rc) rc = upload_scalars(c, d);
  if (rc) return rc;
  return kick_eager(c, in, out);
}

// Timing of a finished step: drift (ev5..ev6) and the whole step (ev5..ev7).
static void step_times(cube_ctx* c, cube_step_out* out) {
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]);
  out->tcat[0] = ms;
  out->tcat[5] += ms;
  ms = 0;
  cudaEventElapsedTime(&ms, c->ev[5], c->ev[7]);
  out->tcat[6] = ms;  // whole step on the device, host gaps included
}

// One step as one CUDA graph (cube_params.step_graph): scalars up, drift, PM1, PM2,
// classes, device-built class lists, PM3, PP, momentum and the results copied back, with
// no host synchronisation inside.  The PM3 chunks are laid out for the previous step's
// class histogram with headroom.  When a step's classes outgrow them, the graph kicks the
// particles of the listed subtiles and skips PP (device flag); the host then runs PM3 for
// the unlisted subtiles and PP, which gives every particle the same operations in the
// same order as the eager step.  Graphs are kept per particle-buffer parity, particle
// count and plan, and captured on first use.
static int step_graph(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  StepDev d;
  int rc = make_scalars(c, in, true, d);
  if (rc) return rc;
  if (!c->have_est) {  // first step: classes of the current state
    CK(cudaMemsetAsync(c->napm, 0, 32, c->s));
    LAUNCH(c, K_CLASSIFY, 1, k_classify<<<nblk(c->ns3), 256, 0, c->s>>>(c->G, c->rhoc, c->ns3, c->ires, c->napm));
    CK(cudaMemcpyAsync(c->napm_est, c->napm, 32, cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    c->have_est = true;
  }
  const PM3Plan pl = make_plan(c, c->napm_est, true);
  rc = ensure_plan_buffers(c, pl);
  if (rc) return rc;
  const bool ppq = c->P.pp_queue && c->P.pp_on;
  PPShape pps;
  if (ppq) {
    if (c->maxcount_est < 0) {  // occupancy of the current state
      CK(cudaMemsetAsync(&c->rdev->maxcount, 0, 4, c->s));
      k_ppq_maxcount<<<(unsigned)std::min<int64_t>(nblk(c->G.ncells), 4 * c->nsm), 256, 0, c->s>>>(
          c->cstart, c->G.c0, c->G.c1, &c->rdev->maxcount);
      ++c->launches;
      CK(cudaMemcpyAsync(&c->maxcount_est, &c->rdev->maxcount, 4, cudaMemcpyDeviceToHost, c->s));
      CK(cudaStreamSynchronize(c->s));
    }
    rc = pp_shape(c, c->maxcount_est, pps);
    if (rc) return rc;
  }
  for (int cl = 2; cl <= 5; ++cl)
    if (pl.cap[cl] > 0 && !kernel_table(c, 3, cl)) return CUBE_E_CUDA;  // tables exist before any capture
  if (!kernel_table(c, 1, 0) || !kernel_table(c, 2, 0)) return CUBE_E_CUDA;
  const int parity = c->xp == c->xp_base ? 0 : 1;
  StepGraph* g = nullptr;
  for (auto& x : c->graphs)
    if (x.parity == parity && x.np == c->np && x.prof == c->prof && same_plan(x.plan, pl) && x.pps == pps) g = &x;
  if (!g) {
    // one graph per parity: a new plan replaces the old one of this parity
    for (size_t i = 0; i < c->graphs.size(); ++i)
      if (c->graphs[i].parity == parity) {
        CK(cudaStreamSynchronize(c->s));
        cudaGraphExecDestroy(c->graphs[i].exec);
        for (cudaEvent_t e : c->graphs[i].events) cudaEventDestroy(e);
        c->graphs.erase(c->graphs.begin() + i);
        break;
      }
    StepGraph ng;
    ng.parity = parity;
    ng.np = c->np;
    ng.plan = pl;
    ng.pps = pps;
    ng.prof = c->prof;
    c->cap_graph = &ng;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeRelaxed));
    cudaMemcpyAsync(c->sd, c->h_sd, sizeof(StepDev), cudaMemcpyHostToDevice, c->s);
    mark(c, c->ev[5]);
    enqueue_drift(c, false);
    swap_drift(c);
    mark(c, c->ev[6]);
    rc = enqueue_kick_a(c);
    if (!rc) rc = enqueue_lists(c, pl);
    if (!rc) rc = enqueue_pm3(c, pl, false);
    if (!rc) {
      mark(c, c->ev[3]);
      enqueue_pp_and_momentum(c, c->overflow, ppq ? &pps : nullptr);
      mark(c, c->ev[7]);
      cudaMemcpyAsync(c->rhost, c->rdev, sizeof(StepRes), cudaMemcpyDeviceToHost, c->s);
    }
    const cudaError_t ce = cudaStreamEndCapture(c->s, &graph);
    swap_drift(c);  // undo: the graph has not run yet
    c->cap_graph = nullptr;
    cudaError_t ie = cudaSuccess;
    if (!rc && ce == cudaSuccess) ie = cudaGraphInstantiate(&ng.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc || ce != cudaSuccess || ie != cudaSuccess) {
      for (cudaEvent_t e : ng.events) cudaEventDestroy(e);
      cudaGetLastError();
      if (rc) return rc;
      return fail(CUBE_E_CUDA, std::string("step graph capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ie));
    }
    c->graphs.push_back(std::move(ng));
    g = &c->graphs.back();
  }
  *c->h_sd = d;
  after_checkpoint_copy(c);
  CK(cudaGraphLaunch(g->exec, c->s));
  CK(cudaStreamSynchronize(c->s));
  swap_drift(c);
  c->launches += g->kernels;
  if (c->prof)
    for (const ProfRec& r : g->recs) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, g->events[r.a], g->events[r.b]) == cudaSuccess) {
        c->prof_ms[r.cls] += ms;
        c->prof_n[r.cls] += 1;
      }
    }
  if (c->rhost->overflow) {
    // the classes outgrew the plan: PM3 of the subtiles beyond each class's capacity, then
    // PP (skipped by the graph).  The f2max, vmax and mass sums of PM3 accumulate over
    // both passes; PP contributed nothing yet; the momentum is recomputed.
    CK(cudaMemsetAsync(c->overflow, 0, 4, c->s));
    int32_t napm[8];
    memcpy(napm, c->rhost->napm, sizeof napm);
    const PM3Plan rest = make_plan(c, napm, false, pl.cap);
    rc = ensure_plan_buffers(c, rest);
    if (!rc) rc = enqueue_lists(c, rest);
    if (!rc) rc = enqueue_pm3(c, rest, false);
    if (rc) return rc;
    CK(mark(c, c->ev[3]));
    enqueue_pp_and_momentum(c, nullptr, ppq ? &pps : nullptr);
    CK(mark(c, c->ev[7]));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->rhost, c->rdev, sizeof(StepRes), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    prof_collect(c);
  }
  memcpy(c->napm_est, c->rhost->napm, sizeof c->napm_est);
  c->maxcount_est = c->rhost->maxcount;
  if (c->rhost->err) {
    CK(cudaMemsetAsync(c->err, 0, 4, c->s));
    CK(cudaStreamSynchronize(c->s));
    return err_code(c->rhost->err);
  }
  if (c->rhost->total != c->np) return fail(CUBE_E_COUNT, "drift: particle count not conserved");
  if (out) {
    fill_out(c, in, out);
    step_times(c, out);
  }
  return 0;
}

int cube_gpu_step(cube_ctx* c, const cube_step_in* in, cube_step_out* out) {
  if (!c || !in) return fail(CUBE_E_ARG, "null argument");
  if (!c->loaded) return fail(CUBE_E_STATE, "step before upload");
  CK(cudaSetDevice(c->device));
  // graph replay unless a test capture is armed (it copies with host-side allocations); a
  // split run steps eagerly (its collectives run on the host between the stages)
  if (c->P.step_graph && c->cap_level == 0 && c->G.nslab == 1) return step_graph(c, in, out);
  StepDev d;
  int rc = make_scalars(c, in, true, d);
  if (!rc) rc = upload_scalars(c, d);
  if (rc) return rc;
  // ev[5]: step start, ev[6]: drift end, ev[7]: step end (all on the context stream)
  CK(cudaEventRecord(c->ev[5], c->s));
  if (c->G.nslab > 1) {  // ghosts, drift, the count check over the slabs, then the kick
    if (!c->ghosts) rc = slab_exchange(c);
    if (rc) return rc;
    const int64_t nown = c->own1 - c->own0;
    enqueue_drift(c, false);
    CK(cudaGetLastError());
    swap_drift(c);
    CK(cudaEventRecord(c->ev[6], c->s));
    int64_t total = 0;
    CK(cudaMemcpyAsync(&total, c->total, 8, cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    rc = slab_after_drift(c, nown, total);
    if (!rc) rc = kick_eager(c, in, out);
    CK(cudaEventRecord(c->ev[7], c->s));
    CK(cudaEventSynchronize(c->ev[7]));
    if (rc) return rc;
    if (out) step_times(c, out);
    return 0;
  }
  enqueue_drift(c, false);
  CK(cudaGetLastError());
  swap_drift(c);
  CK(cudaEventRecord(c->ev[6], c->s));
  rc = kick_eager(c, in, out);
  CK(cudaEventRecord(c->ev[7], c->s));
  CK(cudaEventSynchronize(c->ev[7]));
  if (rc) return rc;
  if (c->rhost->total != c->np) return fail(CUBE_E_COUNT, "drift: particle count not conserved");
  if (out) step_times(c, out);
  return 0;
}

// One step on a host-resident particle state: upload, drift, kick, download, with the
// copies that the step does not wait for moved onto a side stream.  Positions,
// velocities and cell counts go up first; the ids follow on the side stream while the
// drift runs (its gather leaves them alone) and are put in the drift's order there by
// k_permute_ids; the drift's outputs (positions, ids, cell counts) come down on that
// stream during the kick, which only reads them; the velocities come down after the
// kick.  Same results as cube_gpu_upload + cube_gpu_step + cube_gpu_download on the
// same arrays.
int cube_gpu_step_host(cube_ctx* c, const cube_step_in* in, cube_step_out* out, void* xp, float* vp, int64_t* pid,
                       int32_t* rhoc, int64_t nplocal) {
  if (!c || !in || !xp || !vp || !pid || !rhoc || nplocal <= 0) return fail(CUBE_E_ARG, "bad step_host arguments");
  CK(cudaSetDevice(c->device));
  const Geo& G = c->G;
  if (G.nslab > 1)  // the arrays hold nplocal particles, and a split run's count changes in the step
    return fail(CUBE_E_ARG, "cube_gpu_step_host takes nslab = 1; split runs use upload, step and download");
  if (!c->s2) {
    CK(cudaStreamCreateWithFlags(&c->s2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_drift, cudaEventDisableTiming));
  }
  // the copies the host arrays still feed must be done before the arrays are checked
  // or reused by a failed call
  auto drain = [&]() {
    cudaStreamSynchronize(c->s2);
    cudaStreamSynchronize(c->s);
  };
  StepDev d;
  int rc = make_scalars(c, in, true, d);
  if (!rc) rc = alloc_particles(c, nplocal);
  if (rc) return rc;
  c->np = nplocal;
  c->loaded = false;
  after_checkpoint_copy(c);
  CK(cudaMemcpyAsync(c->rhoc, rhoc, (size_t)G.ncells * 4, cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->xp, xp, (size_t)nplocal * 3 * c->xbytes, cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->vp, vp, (size_t)nplocal * 12, cudaMemcpyHostToDevice, c->s));
  // the ids go up after the arrays the drift starts with (not sharing the link with
  // them) and are permuted on the side stream once the drift is done
  CK(cudaEventRecord(c->ev_up, c->s));
  CK(cudaStreamWaitEvent(c->s2, c->ev_up, 0));
  CK(cudaMemcpyAsync(c->pid, pid, (size_t)nplocal * 8, cudaMemcpyHostToDevice, c->s2));
  // the cell counts are validated on the host while the copies run
  int64_t sum = 0;
  bool neg = false;
  for (int64_t i = 0; i < G.ncells; ++i) {
    neg |= rhoc[i] < 0;
    sum += rhoc[i];
  }
  if (neg || sum != nplocal) {
    drain();
    return neg ? fail(CUBE_E_ARG, "negative rhoc") : fail(CUBE_E_COUNT, "sum(rhoc) != nplocal");
  }
  LAUNCH(c, K_SCAN, 3, exclusive_scan(c->rhoc, c->cstart, G.ncells, c->scan_tmp, c->s));
  LAUNCH(c, K_FILL, 1, k_fill_pcell<<<nblk(G.ncells), 256, 0, c->s>>>(c->cstart, G.ncells, c->pcell));
  CK(cudaGetLastError());
  c->loaded = true;
  rc = upload_scalars(c, d);
  if (rc) {
    drain();
    return rc;
  }
  CK(cudaEventRecord(c->ev[5], c->s));
  enqueue_drift(c, true);
  CK(cudaGetLastError());
  swap_drift(c);
  CK(cudaEventRecord(c->ev[6], c->s));
  CK(cudaEventRecord(c->ev_drift, c->s));
  CK(cudaStreamWaitEvent(c->s2, c->ev_drift, 0));
  CK(cudaMemcpyAsync(xp, c->xp, (size_t)c->np * 3 * c->xbytes, cudaMemcpyDeviceToHost, c->s2));
  CK(cudaMemcpyAsync(rhoc, c->rhoc, (size_t)G.ncells * 4, cudaMemcpyDeviceToHost, c->s2));
  k_permute_ids<<<nblk(c->np), 256, 0, c->s2>>>(c->np, c->ssrc, c->pid2, c->pid);  // after the id upload (s2 order)
  CK(cudaGetLastError());
  ++c->launches;
  CK(cudaMemcpyAsync(pid, c->pid, (size_t)c->np * 8, cudaMemcpyDeviceToHost, c->s2));
  rc = kick_eager(c, in, out);
  CK(cudaEventRecord(c->ev[7], c->s));
  if (!rc) CK(cudaMemcpyAsync(vp, c->vp, (size_t)c->np * 12, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  CK(cudaStreamSynchronize(c->s2));
  if (!rc && c->rhost->total != c->np) rc = fail(CUBE_E_COUNT, "drift: particle count not conserved");
  if (rc) c->loaded = false;
  if (!rc && out) step_times(c, out);
  return rc;
}

int cube_gpu_pp_shape(cube_ctx* c, int cls, int T, int B, int J) {
  if (!c || cls < 0 || cls > 3) return fail(CUBE_E_ARG, "bad PP class");
  if (T <= 0) {
    c->pp_tuned[cls] = false;
    return 0;
  }
  if (B != 32 && B != 64 && B != 128 && B != 256 && B != 512)
    return fail(CUBE_E_ARG, "PP item size B must be 32, 64, 128, 256 or 512");
  if (J < 32 || J > 4096) return fail(CUBE_E_ARG, "PP chunk J must be in 32..4096");
  PPShape sh;
  sh.T = T;
  sh.B = B;
  sh.J = J;
  c->pp_best[cls] = sh;
  c->pp_tuned[cls] = true;
  c->pp_tune_ms[cls] = 0;
  return 0;
}

int cube_gpu_pp_shape_get(cube_ctx* c, int cls, int* T, int* B, int* J, double* ms) {
  if (!c || cls < 0 || cls > 3) return fail(CUBE_E_ARG, "bad PP class");
  if (!c->pp_tuned[cls]) return 0;
  if (T) *T = c->pp_best[cls].T;
  if (B) *B = c->pp_best[cls].B;
  if (J) *J = c->pp_best[cls].J;
  if (ms) *ms = c->pp_tune_ms[cls];
  return 1;
}

int cube_gpu_profile(cube_ctx* c, int enable) {
  if (!c) return fail(CUBE_E_ARG, "null context");
  CK(cudaStreamSynchronize(c->s));
  prof_collect(c);
  c->prof = enable != 0;
  for (int i = 0; i < K_NCLASS; ++i) {
    c->prof_ms[i] = 0;
    c->prof_n[i] = 0;
  }
  return 0;
}

int cube_gpu_profile_read(cube_ctx* c, double* ms, int64_t* count, int n) {
  if (!c) return fail(CUBE_E_ARG, "null context");
  for (int i = 0; i < n && i < K_NCLASS; ++i) {
    if (ms) ms[i] = c->prof_ms[i];
    if (count) count[i] = c->prof_n[i];
  }
  return K_NCLASS;
}

const char* cube_gpu_profile_name(int i) { return (i >= 0 && i < K_NCLASS) ? KNAMES[i] : ""; }

int64_t cube_gpu_kernel_launches(cube_ctx* c) { return c ? c->launches : -1; }

int cube_gpu_capture(cube_ctx* c, int level, int box, int what) {
  if (!c) return fail(CUBE_E_ARG, "null context");
  c->cap_level = level;
  c->cap_box = box;
  c->cap_what = what;
  return 0;
}

int cube_gpu_captured(cube_ctx* c, float* out, int64_t n) {
  if (!c || !out) return fail(CUBE_E_ARG, "null argument");
  if (!c->cap_buf) return fail(CUBE_E_STATE, "nothing captured");
  CK(cudaSetDevice(c->device));
  const bool is_int = c->cap_n < 0;
  const int64_t m = is_int ? -c->cap_n : c->cap_n;
  if (n < m) return fail(CUBE_E_ARG, "capture buffer too small");
  if (is_int) {
    std::vector<long long> h(m);
    CK(cudaMemcpy(h.data(), c->cap_buf, m * 8, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < m; ++i) out[i] = (float)std::ldexp((double)h[i], -40) * c->G.mass_p;
  } else {
    std::vector<float> h(m);
    CK(cudaMemcpy(h.data(), c->cap_buf, m * 4, cudaMemcpyDeviceToHost));
    // density captures hold unscaled weights; phi captures are final
    const float sc = (c->cap_what == 0) ? c->G.mass_p : 1.f;
    for (int64_t i = 0; i < m; ++i) out[i] = (c->cap_what == 0) ? h[i] * sc : h[i];
  }
  return (int)m;
}

int cube_gpu_ic(cube_ctx* c, const cube_ic_in* in, cube_ic_out* out) {
  if (!c || !in || !in->pk_k || !in->pk_p || in->npk < 2 || in->nic < 1) return fail(CUBE_E_ARG, "bad IC arguments");
  if (c->G.nslab > 1) return fail(CUBE_E_ARG, "cube_gpu_ic generates the whole box: nslab must be 1");
  CK(cudaSetDevice(c->device));
  const Geo& G = c->G;
  const int nw = in->nic * G.ng;
  const int nlat = G.nc * (int)c->P.np_nc;
  if ((G.rcs * in->nic) % (int)c->P.np_nc) return fail(CUBE_E_ARG, "ratio_cs*nic must be a multiple of np_nc");
  const int64_t np = (int64_t)nlat * nlat * nlat;
  int rc = alloc_particles(c, np);
  if (!rc) rc = add_fft(c, nw);
  if (rc) return rc;
  // mesh: the arena when it is large enough, else a temporary buffer
  const Pitch pt = pitch_of(c, nw, false);
  const size_t mbytes = mesh_bytes(c, nw, 1, false);
  void* mesh = c->arena;
  void* tmp_mesh = nullptr;
  if (mbytes > c->arena_bytes) {
    CK(cudaMalloc(&tmp_mesh, mbytes));
    mesh = tmp_mesh;
  }
  std::vector<double> hk(in->npk), hp(in->npk);
  for (int i = 0; i < in->npk; ++i) {
    if (!(in->pk_k[i] > 0) || !(in->pk_p[i] > 0)) {
      if (tmp_mesh) cudaFree(tmp_mesh);
      return fail(CUBE_E_ARG, "P(k) table must be positive");
    }
    hk[i] = std::log(in->pk_k[i]);
    hp[i] = std::log(in->pk_p[i]);
  }
  float* gtab = nullptr;
  double *lk = nullptr, *lp = nullptr;
  const int64_t gcount = (int64_t)nw * nw * (nw / 2 + 1);
  CK(cudaMalloc(&gtab, gcount * sizeof(float)));
  CK(cudaMalloc(&lk, in->npk * sizeof(double)));
  CK(cudaMalloc(&lp, in->npk * sizeof(double)));
  CK(cudaMemcpyAsync(lk, hk.data(), in->npk * sizeof(double), cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(lp, hp.data(), in->npk * sizeof(double), cudaMemcpyHostToDevice, c->s));
  CK(cudaMemsetAsync(mesh, 0, mbytes, c->s));
  const uint2 key = make_uint2((uint32_t)in->seed, (uint32_t)(in->seed >> 32));
  const int64_t npair = (int64_t)nw * nw * nw / 2;
  LAUNCH(c, K_FILL, 1, k_ic_noise<<<nblk(npair), 256, 0, c->s>>>((float*)mesh, nw, pt.pr, pt.plr, key));
  LAUNCH(c, K_GREEN, 1, k_ic_multiplier<<<nblk(gcount), 256, 0, c->s>>>(gtab, nw, c->P.box, lk, lp, in->npk));
  float* phi = (float*)mesh;
  launch_fft(c, nw, 1, mesh, false, 1.f, phi, (float2*)mesh, gtab, (float)nw, 3, 1);
  ICArgs A;
  A.nw = nw;
  A.nlat = nlat;
  A.step = G.rcs * in->nic / (int)c->P.np_nc;
  A.np_nc = (int)c->P.np_nc;
  A.nic = in->nic;
  A.vf = in->vfactor;
  A.lat_off = (0.5 / in->nic) / G.rcs;
  CK(cudaMemsetAsync(c->red, 0, 64 * sizeof(float), c->s));
  LAUNCH(c, K_FILL, 1, k_ic_gradmax<<<nblk(np), 256, 0, c->s>>>(phi, pt.pf, pt.plf, A, c->red));
  float gm[3];
  CK(cudaMemcpyAsync(gm, c->red, sizeof(gm), cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  // reference grad_max is |phi(i)-phi(i+2)| on the IC grid; the corner gradient is half of it
  const double PI = 3.141592653589793;
  for (int d = 0; d < 3; ++d) gm[d] *= 2.f;
  A.nlayer = 2 * (int)std::ceil(gm[2] * A.np_nc / (8.0 * A.nic * PI * G.rcs)) + 3;  // ic.f90:587
  CK(cudaMemsetAsync(c->rhoc2, 0, G.ncells * 4, c->s));
  CK(cudaMemsetAsync(c->fill, 0, G.ncells * 4, c->s));
  CK(cudaMemsetAsync(c->nbig, 0, 8, c->s));
  LAUNCH(c, K_FILL, 1, k_ic_particles<<<nblk(np), 256, 0, c->s>>>(G, phi, pt.pf, pt.plf, A, c->xp, c->vp, c->pid, c->dest,
                                                                  c->key, c->rhoc2, c->err));
  LAUNCH(c, K_SCAN, 3, exclusive_scan(c->rhoc2, c->cstart2, G.ncells, c->scan_tmp, c->s));
  LAUNCH(c, K_DRIFT_SCATTER, 1, k_drift_scatter<<<nblk(np), 256, 0, c->s>>>(np, c->dest, c->key, c->cstart2, c->fill, c->skey, c->ssrc));
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_sort_small<<<nblk((G.ncells + 1) / 2 * 32), 256, 0, c->s>>>(G.ncells, c->rhoc2, c->cstart2, c->skey,
                                                                                     c->ssrc, c->biglist, c->nbig));
  const int max_seg = c->P.max_segment > 0 ? std::min(c->P.max_segment, 16384) : 16384;
  const unsigned nbb = (unsigned)std::min<int64_t>(G.ncells, c->nsm);
  LAUNCH(c, K_DRIFT_SORT, 1, k_drift_sort_big<<<nbb, 512, drift_sort_smem(max_seg), c->s>>>(
                                 c->biglist, c->nbig, c->rhoc2, c->cstart2, c->skey, c->ssrc, max_seg, c->hugelist,
                                 c->nbig + 1));
  enqueue_huge_sort(c);
  c->np = np;
  CK(cudaMemsetAsync(c->sd, 0, sizeof(StepDev), c->s));  // dt_mid = 0: the gather only sorts
  LAUNCH(c, K_DRIFT_GATHER, 1, k_drift_gather<<<nblk(np), 256, 0, c->s>>>(G, np, c->ssrc, c->dest, c->xp, c->vp, c->pid, c->sd,
                                                                         c->xp2, c->vp2, c->pid2, c->pcell2, nullptr));
  CK(cudaGetLastError());
  rc = check_err(c);
  cudaFree(gtab);
  cudaFree(lk);
  cudaFree(lp);
  if (tmp_mesh) cudaFree(tmp_mesh);
  if (rc) return rc;
  std::swap(c->xp, c->xp2);
  std::swap(c->vp, c->vp2);
  std::swap(c->pid, c->pid2);
  std::swap(c->pcell, c->pcell2);
  std::swap(c->rhoc, c->rhoc2);
  std::swap(c->cstart, c->cstart2);
  c->loaded = true;
  c->have_est = false;
  c->maxcount_est = -1;
  prof_collect(c);
  if (out) {
    memset(out, 0, sizeof(*out));
    out->nplocal = np;
    float vm = 0.f;
    for (int d = 0; d < 3; ++d) {
      out->grad_max[d] = gm[d];
      out->vmax[d] = (float)(gm[d] / (8.0 * A.nic * PI) * in->vfactor);
      vm = std::max(vm, std::fabs(out->vmax[d]));
    }
    out->vz_max = out->vmax[2];
    out->dt_vmax = 0.9f * 16.f / vm;
    out->nlayer = A.nlayer;
    out->mass_p_cdm = (float)((double)G.ng * G.ng * G.ng / (double)np);
  }
  return 0;
}

// ZIPV codec on host arrays, computed on the context's device.
static int zipv_run(cube_ctx* c, const void* in, void* out, int64_t n, float sigma_vi, bool encode) {
  if (!c || !in || !out || n < 0) return fail(CUBE_E_ARG, "bad zipv arguments");
  if (!(sigma_vi > 0.f)) return fail(CUBE_E_ARG, "sigma_vi must be positive");
  if (n == 0) return 0;
  CK(cudaSetDevice(c->device));
  void *din = nullptr, *dout = nullptr;
  const size_t bin = encode ? 4 : 2, bout = encode ? 2 : 4;
  CK(cudaMalloc(&din, n * bin));
  CK(cudaMalloc(&dout, n * bout));
  CK(cudaMemcpyAsync(din, in, n * bin, cudaMemcpyHostToDevice, c->s));
  if (encode)
    LAUNCH(c, K_FILL, 1, k_zipv_encode<<<nblk(n), 256, 0, c->s>>>((const float*)din, (int16_t*)dout, n, sigma_vi));
  else
    LAUNCH(c, K_FILL, 1, k_zipv_decode<<<nblk(n), 256, 0, c->s>>>((const int16_t*)din, (float*)dout, n, sigma_vi));
  CK(cudaMemcpyAsync(out, dout, n * bout, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  cudaFree(din);
  cudaFree(dout);
  return 0;
}

int cube_gpu_zipv_encode(cube_ctx* c, const float* v, int16_t* code, int64_t n, float sigma_vi) {
  return zipv_run(c, v, code, n, sigma_vi, true);
}

int cube_gpu_zipv_decode(cube_ctx* c, const int16_t* code, float* v, int64_t n, float sigma_vi) {
  return zipv_run(c, code, v, n, sigma_vi, false);
}

int cube_gpu_download_zipv(cube_ctx* c, void* xp, int16_t* vp_code, int64_t* pid, int32_t* rhoc, int64_t* nplocal,
                           float sigma_vi) {
  if (!c || !c->loaded) return fail(CUBE_E_STATE, "no particles on device");
  if (!(sigma_vi > 0.f)) return fail(CUBE_E_ARG, "sigma_vi must be positive");
  CK(cudaSetDevice(c->device));
  int16_t* dcode = nullptr;
  CK(cudaMalloc(&dcode, (size_t)c->np * 3 * 2));
  LAUNCH(c, K_FILL, 1, k_zipv_encode<<<nblk(c->np * 3), 256, 0, c->s>>>(c->vp, dcode, c->np * 3, sigma_vi));
  if (vp_code) CK(cudaMemcpyAsync(vp_code, dcode, (size_t)c->np * 6, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  cudaFree(dcode);
  return cube_gpu_download(c, xp, nullptr, pid, rhoc, nplocal);
}

int cube_gpu_int2real(cube_ctx* c, float* xv, int64_t n) {
  if (!c || !xv) return fail(CUBE_E_ARG, "null argument");
  if (!c->loaded) return fail(CUBE_E_STATE, "int2real before upload");
  if (n < 3 * c->np) return fail(CUBE_E_ARG, "xv needs 3*nplocal floats");
  CK(cudaSetDevice(c->device));
  float* d = nullptr;
  CK(cudaMalloc(&d, (size_t)c->np * 3 * sizeof(float)));
  LAUNCH(c, K_FILL, 1, k_int2real<<<nblk(c->np), 256, 0, c->s>>>(c->G, c->np, c->xp, c->pcell, d));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(xv, d, (size_t)c->np * 3 * sizeof(float), cudaMemcpyDeviceToHost, c->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->s);
  cudaFree(d);
  if (e != cudaSuccess) return fail(CUBE_E_CUDA, std::string("int2real: ") + cudaGetErrorString(e));
  return 0;
}

int cube_gpu_green_table(cube_ctx* c, int level, int iapm, float* out, int64_t n) {
  if (!c || !out) return fail(CUBE_E_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const Geo& G = c->G;
  float* src = nullptr;
  int m = 0;
  if (level == 1) { src = c->green1; m = G.nc; }
  else if (level == 2) { src = c->green2; m = G.ngt; }
  else if (level == 3 && iapm >= 2 && iapm <= 5) { src = green3(c, iapm); m = G.nft[iapm]; }
  if (!src) return fail(CUBE_E_ARG, "bad level/iapm");
  const int64_t cnt = (int64_t)m * m * (m / 2 + 1);
  if (n < cnt) return fail(CUBE_E_ARG, "buffer too small");
  CK(cudaStreamSynchronize(c->s));
  CK(cudaMemcpy(out, src, cnt * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int cube_gpu_checkpoint_wait(cube_ctx* c) {
  if (!c) return fail(CUBE_E_ARG, "null context");
  if (c->ck_thread.joinable()) c->ck_thread.join();
  c->ckpt_pending = false;
  const int st = c->ck_status;
  c->ck_status = 0;
  if (st) return fail(st, c->ck_error);
  return 0;
}

int cube_gpu_checkpoint_async(cube_ctx* c, const cube_ckpt_files* files, const void* header, int64_t header_bytes) {
  if (!c || !files || !files->info || !files->xp || !files->vp || !files->np || !files->id || !header ||
      header_bytes <= 0)
    return fail(CUBE_E_ARG, "bad checkpoint arguments");
  if (!c->loaded) return fail(CUBE_E_STATE, "checkpoint before upload");
  int rc = cube_gpu_checkpoint_wait(c);  // one checkpoint in flight at a time
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  if (!c->s3) {
    CK(cudaStreamCreateWithFlags(&c->s3, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_ckpt, cudaEventDisableTiming));
  }
  const Geo& G = c->G;
  // this rank's particles (a split run's store may also hold ghosts)
  const bool slabs = G.nslab > 1;
  const int64_t o = slabs ? c->own0 : 0, n = slabs ? c->own1 - c->own0 : c->np;
  const size_t bx = (size_t)n * 3 * c->xbytes, bv = (size_t)n * 12, bn = (size_t)G.ncells * 4, bi = (size_t)n * 8;
  const size_t need = bx + bv + bn + bi + 64;
  if (need > c->ck_bytes) {
    if (c->ck_host) cudaFreeHost(c->ck_host);
    c->ck_host = nullptr;
    c->ck_bytes = 0;
    CK(cudaMallocHost(&c->ck_host, need));
    c->ck_bytes = need;
  }
  char* hx = static_cast<char*>(c->ck_host);
  char* hv = hx + bx;
  char* hn = hv + bv;
  char* hi = hn + bn;
  // the state as the context stream leaves it, copied on the side stream
  CK(cudaEventRecord(c->ev_ckpt, c->s));
  CK(cudaStreamWaitEvent(c->s3, c->ev_ckpt, 0));
  CK(cudaMemcpyAsync(hx, (char*)c->xp + o * 3 * c->xbytes, bx, cudaMemcpyDeviceToHost, c->s3));
  CK(cudaMemcpyAsync(hv, c->vp + 3 * o, bv, cudaMemcpyDeviceToHost, c->s3));
  CK(cudaMemcpyAsync(hn, c->rhoc, bn, cudaMemcpyDeviceToHost, c->s3));
  CK(cudaMemcpyAsync(hi, c->pid + o, bi, cudaMemcpyDeviceToHost, c->s3));
  CK(cudaEventRecord(c->ev_ckpt, c->s3));
  c->ckpt_pending = true;
  struct Part {
    std::string path;
    const char* data;
    size_t bytes;
  };
  std::vector<Part> parts = {{files->info, static_cast<const char*>(header), (size_t)header_bytes},
                             {files->xp, hx, bx}, {files->vp, hv, bv}, {files->np, hn, bn}, {files->id, hi, bi}};
  std::vector<char> hdr(static_cast<const char*>(header), static_cast<const char*>(header) + header_bytes);
  const int dev = c->device;
  cudaEvent_t ev = c->ev_ckpt;
  c->ck_status = 0;
  c->ck_error.clear();
  const int64_t c0 = G.c0, c1 = G.c1, ncells = G.ncells;
  c->ck_thread = std::thread([c, parts, hdr, dev, ev, slabs, hn, c0, c1, ncells]() mutable {
    parts[0].data = hdr.data();  // the caller's header may go away once the call returns
    cudaSetDevice(dev);
    if (cudaEventSynchronize(ev) != cudaSuccess) {
      c->ck_status = CUBE_E_CUDA;
      c->ck_error = "checkpoint copies failed";
      return;
    }
    if (slabs) {  // ghost cells are other ranks' particles
      memset(hn, 0, (size_t)c0 * 4);
      memset(hn + c1 * 4, 0, (size_t)(ncells - c1) * 4);
    }
    for (const Part& p : parts) {
      FILE* f = fopen(p.path.c_str(), "wb");
      if (!f || fwrite(p.data, 1, p.bytes, f) != p.bytes || fclose(f) != 0) {
        c->ck_status = CUBE_E_ARG;
        c->ck_error = "checkpoint: cannot write " + p.path;
        return;
      }
    }
  });
  return 0;
}

int cube_gpu_nu_transfer(cube_ctx* c, const float* kh_log, const float* tf_log, int nb) {
  if (!c || nb < 0 || (nb > 0 && (!kh_log || !tf_log))) return fail(CUBE_E_ARG, "bad neutrino transfer arguments");
  if (nb > 0 && nb < 3) return fail(CUBE_E_ARG, "the transfer table needs at least three points");
  for (int i = 1; i < nb; ++i)
    if (!(kh_log[i] > kh_log[i - 1])) return fail(CUBE_E_ARG, "log k of the transfer table must increase");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->s));  // the previous table may still be read
  // captured steps name the force kernels: the Green tables or, with neutrinos, the
  // rescaled copies (rebuilt in place before each step); switching between the two
  // needs new captures
  const bool before = c->P.f_nu > 0.f || c->nu_nb >= 3, after = c->P.f_nu > 0.f || nb >= 3;
  if (before != after) drop_graphs(c);
  if (c->nu_tab) cudaFree(c->nu_tab);
  c->nu_tab = nullptr;
  c->nu_nb = 0;
  if (nb > 0) {
    CK(cudaMalloc(&c->nu_tab, (size_t)2 * nb * sizeof(float)));
    CK(cudaMemcpy(c->nu_tab, kh_log, nb * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->nu_tab + nb, tf_log, nb * sizeof(float), cudaMemcpyHostToDevice));
    c->nu_nb = nb;
  }
  ++c->nu_ver;
  return 0;
}

int cube_gpu_kernel_table(cube_ctx* c, int level, int iapm, float* out, int64_t n) {
  if (!c || !out) return fail(CUBE_E_ARG, "null argument");
  if (level < 1 || level > 3 || (level == 3 && (iapm < 2 || iapm > 5))) return fail(CUBE_E_ARG, "bad level/iapm");
  CK(cudaSetDevice(c->device));
  const Geo& G = c->G;
  const int m = level == 1 ? G.nc : level == 2 ? G.ngt : G.nft[iapm];
  const int64_t cnt = (int64_t)m * m * (m / 2 + 1);
  if (n < cnt) return fail(CUBE_E_ARG, "buffer too small");
  const float* src = kernel_table(c, level, iapm);
  if (!src) return CUBE_E_CUDA;
  CK(cudaStreamSynchronize(c->s));
  CK(cudaMemcpy(out, src, cnt * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int cube_gpu_set_comm(cube_ctx* c, const cube_comm* comm) {
  if (!c || !comm || !comm->allreduce || !comm->sendrecv) return fail(CUBE_E_ARG, "cube_gpu_set_comm: null callback");
  c->comm = *comm;
  c->have_comm = true;
  return 0;
}

int64_t cube_slab_cells(const cube_params* p, int which, int64_t* out, int64_t n) {
  if (!p || which < 0 || which > 4 || n < 0) return fail(CUBE_E_ARG, "bad cube_slab_cells arguments");
  if (p->ratio_cs <= 0 || p->nnt <= 0 || p->ng % p->ratio_cs || (p->ng / p->ratio_cs) % p->nnt)
    return fail(CUBE_E_ARG, "ng, ratio_cs, nnt must divide evenly");
  const int nslab = p->nslab > 1 ? p->nslab : 1;
  if (p->nnt % nslab || (nslab > 1 && (p->slab < 0 || p->slab >= nslab)))
    return fail(CUBE_E_ARG, "nslab must divide nnt, and 0 <= slab < nslab");
  const Geo G = make_geo(*p);
  if (G.ncb > G.nt) return fail(CUBE_E_ARG, "ghost layers deeper than a tile");
  if (which == 0) {
    const int64_t m = G.c1 - G.c0;
    for (int64_t i = 0; i < m && i < n && out; ++i) out[i] = G.c0 + i;
    return m;
  }
  if (nslab == 1) return 0;  // one slab: periodic, no layers to exchange
  int tz, lz0;
  slab_layer(G, which - 1, tz, lz0);
  const int64_t nlay = (int64_t)G.nnt * G.nnt * G.ncb * G.nt * G.nt;
  for (int64_t i = 0; i < nlay && i < n && out; ++i) out[i] = layer_cell(G, tz, lz0, i);
  return nlay;
}

int cube_gpu_subtile_class(cube_ctx* c, int32_t* ires, int64_t n) {
  if (!c || !ires || n < c->ns3) return fail(CUBE_E_ARG, "bad argument");
  CK(cudaSetDevice(c->device));
  CK(cudaMemsetAsync(c->napm, 0, 32, c->s));
  LAUNCH(c, K_CLASSIFY, 1, k_classify<<<nblk(c->ns3), 256, 0, c->s>>>(c->G, c->rhoc, c->ns3, c->ires, c->napm));
  CK(cudaMemcpyAsync(ires, c->ires, c->ns3 * 4, cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  return 0;
}

}  // extern "C"

// =================================================================================
// PM1 coarse density with no device allocation (no counterpart in the reference).
//
// Some callers cannot call cudaMalloc when they want a density field: a process whose
// device memory is already held by another framework's caching pool (cudaMalloc then
// fails, or splits memory the pool expects to own), or a caller on a latency-bound path
// where cudaMalloc/cudaFree would synchronise the whole device.  For them
// cube_gpu_pm1_density_noalloc runs the PM1 deposit (particle_mesh.f90 PM1 density)
// with all of its scratch -- cell starts, the scan's tile sums, the per-particle cell
// index and the int64 fixed-point accumulator -- in one file-scope device array sized
// for CUBE_NOALLOC_MAX_CELLS coarse cells and CUBE_NOALLOC_MAX_PARTICLES particles.
// Every device that loads this library holds that array (about 12 MB) until exit.
// =================================================================================
namespace {

constexpr size_t na_round(size_t b) { return (b + 255) / 256 * 256; }
constexpr int64_t kNaCells = CUBE_NOALLOC_MAX_CELLS;
constexpr int64_t kNaParticles = CUBE_NOALLOC_MAX_PARTICLES;
constexpr size_t kNaAccOff = 0;                                                   // int64 [cells]
constexpr size_t kNaStartOff = kNaAccOff + na_round(kNaCells * 8);               // int64 [cells+1]
constexpr size_t kNaScanOff = kNaStartOff + na_round((kNaCells + 1) * 8);        // int64 [tiles+2]
constexpr size_t kNaCellOff = kNaScanOff + na_round(((kNaCells + SCAN_TILE - 1) / SCAN_TILE + 2) * 8);  // int32 [np]
constexpr size_t kNaFlagOff = kNaCellOff + na_round(kNaParticles * 4);           // uint32: negative count seen
constexpr size_t kNaBytes = kNaFlagOff + 256;

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {

// Device address of g_noalloc_scratch per device.  In host code the array's name is only
// a host-side stand-in, so the address is looked up once per device (with that device
// current) and handed to the kernels.
constexpr int kNaMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[kNaMaxDevices];

int noalloc_scratch(unsigned char** out) {
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) return fail(CUBE_E_ARG, "device ordinal beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* a = nullptr;
    CK(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<unsigned char*>(a);
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

// Particle -> cell index from the cell starts; indices at or beyond np are not written,
// so a rhoc that does not sum to np cannot write past the scratch.  A negative count
// (cstart decreasing) raises *bad, which the host turns into CUBE_E_COUNT.
__global__ void k_na_fill_pcell(const int64_t* __restrict__ cstart, int64_t ncells, int64_t np,
                                int32_t* __restrict__ pcell, unsigned* __restrict__ bad) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  if (cstart[c + 1] < cstart[c]) atomicOr(bad, 1u);
  const int64_t b = cstart[c] > 0 ? cstart[c] : 0;
  const int64_t e = cstart[c + 1] < np ? cstart[c + 1] : np;
  for (int64_t i = b; i < e; ++i) pcell[i] = (int32_t)c;
}

// Fixed-point weight sums -> density in mass units, rounded as cube_gpu_captured does.
__global__ void k_na_fixed_to_density(const long long* __restrict__ acc, int64_t n, float mass_p,
                                      float* __restrict__ rho) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rho[i] = __fmul_rn((float)((double)acc[i] * 0x1p-40), mass_p);
}

__global__ void k_na_scale(float* __restrict__ rho, int64_t n, float mass_p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rho[i] = __fmul_rn(rho[i], mass_p);
}

}  // namespace

extern "C" int cube_gpu_pm1_density_noalloc(const cube_params* p, const void* xp, const int32_t* rhoc, int64_t np,
                                            float* rho, void* stream) {
  if (!p || !rhoc || !rho || np < 0 || (np > 0 && !xp)) return fail(CUBE_E_ARG, "null pointer or negative np");
  if (p->ratio_cs <= 0 || p->nnt <= 0 || p->nns <= 0 || p->ng % p->ratio_cs || (p->ng / p->ratio_cs) % p->nnt ||
      ((p->ng / p->ratio_cs) / p->nnt) % p->nns)
    return fail(CUBE_E_ARG, "ng, nnt, nns must divide evenly (parameters.f90:57-59)");
  if (p->izipx != 1 && p->izipx != 2) return fail(CUBE_E_ARG, "izipx must be 1 or 2");
  if (p->mass_p_cdm <= 0.f) return fail(CUBE_E_ARG, "mass_p_cdm must be positive");
  const Geo G = make_geo(*p);
  if (G.ncells > kNaCells || np > kNaParticles) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "cube_gpu_pm1_density_noalloc: %lld coarse cells and %lld particles exceed its static scratch "
             "(at most %lld cells and %lld particles)",
             (long long)G.ncells, (long long)np, (long long)kNaCells, (long long)kNaParticles);
    return fail(CUBE_E_CAPACITY, msg);
  }
  unsigned char* base = nullptr;
  if (int rc = noalloc_scratch(&base)) return rc;
  long long* acc = reinterpret_cast<long long*>(base + kNaAccOff);
  int64_t* cstart = reinterpret_cast<int64_t*>(base + kNaStartOff);
  int64_t* tmp = reinterpret_cast<int64_t*>(base + kNaScanOff);
  int32_t* pcell = reinterpret_cast<int32_t*>(base + kNaCellOff);
  unsigned* bad = reinterpret_cast<unsigned*>(base + kNaFlagOff);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool fixed = p->deposit_mode == CUBE_DEPOSIT_FIXED;
  const int nc = G.nc;
  const int64_t n3 = G.ncells;
  // The array keeps the previous call's contents: clear the accumulator and the cell
  // indices (the scan overwrites every cell start and tile sum it reads).
  if (fixed) CK(cudaMemsetAsync(acc, 0, n3 * 8, s));
  else CK(cudaMemsetAsync(rho, 0, n3 * 4, s));
  if (np > 0) CK(cudaMemsetAsync(pcell, 0, np * 4, s));
  CK(cudaMemsetAsync(bad, 0, sizeof(unsigned), s));
  exclusive_scan(rhoc, cstart, n3, tmp, s);
  k_na_fill_pcell<<<nblk(n3), 256, 0, s>>>(cstart, n3, np, pcell, bad);
  if (np > 0) {
    if (fixed) k_deposit_pm1<true><<<nblk(np), 256, 0, s>>>(G, np, xp, pcell, acc, nc, (int64_t)nc * nc, nullptr);
    else k_deposit_pm1<false><<<nblk(np), 256, 0, s>>>(G, np, xp, pcell, rho, nc, (int64_t)nc * nc, nullptr);
  }
  if (fixed) k_na_fixed_to_density<<<nblk(n3), 256, 0, s>>>(acc, n3, G.mass_p, rho);
  else k_na_scale<<<nblk(n3), 256, 0, s>>>(rho, n3, G.mass_p);
  CK(cudaGetLastError());
  // every particle must belong to a cell (drift.f90:139-143 checks the same sum)
  int64_t total = -1;
  unsigned negative = 0;
  CK(cudaMemcpyAsync(&total, cstart + n3, sizeof total, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&negative, bad, sizeof negative, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (negative) return fail(CUBE_E_COUNT, "rhoc holds a negative count");
  if (total != np) {
    char msg[160];
    snprintf(msg, sizeof msg, "rhoc sums to %lld particles but np is %lld", (long long)total, (long long)np);
    return fail(CUBE_E_COUNT, msg);
  }
  return 0;
}

// =================================================================================
// Power spectrum of the device-resident particles (utilities/cicpower.f90,
// utilities/powerspectrum.f90 auto_power and pk_correction).
// =================================================================================
namespace {

// interp1 (powerspectrum.f90:261-275) as auto_power calls it: the sections xi(2,:) and
// xi(5,:) of xi(10,0:nbin) reach dummies of size nbin, so xdata(i) is bin i-1.
float pk_interp1(const float* xi, int64_t nbin, int rx, int ry, float xq) {
  auto X = [&](int64_t i) { return xi[(i - 1) * 10 + rx]; };
  auto Y = [&](int64_t i) { return xi[(i - 1) * 10 + ry]; };
  int64_t i1 = 1, i2 = nbin;
  while (i2 - i1 > 1) {
    const int64_t im = (i1 + i2) / 2;
    if (xq > X(im)) i1 = im;
    else i2 = im;
  }
  return Y(i1) + (xq - X(i1)) / (X(i2) - X(i1)) * (Y(i2) - Y(i1));
}

// real**integer as gfortran evaluates it (square and multiply).
float pk_powi(float x, int n) {
  float y = (n & 1) ? x : 1.f;
  while (n >>= 1) {
    x = x * x;
    if (n & 1) y = y * x;
  }
  return y;
}

float pk_key_to_float(int k) {
  const int i = k >= 0 ? k : k ^ 0x7fffffff;
  float f;
  memcpy(&f, &i, sizeof f);
  return f;
}

}  // namespace

extern "C" int cube_gpu_power(cube_ctx* c, const cube_power_in* in, float* xi, int64_t nxi, float* delta,
                              cube_power_out* out) {
  if (!c || !in || !xi) return fail(CUBE_E_ARG, "null argument");
  if (!c->loaded) return fail(CUBE_E_STATE, "power spectrum before upload");
  if (c->G.nslab > 1) return fail(CUBE_E_ARG, "cube_gpu_power needs the whole box: nslab must be 1");
  const int nw = in->nw;
  if (nw < 16 || nw > 4096 || !smooth23(nw) || nw % 2)
    return fail(CUBE_E_ARG, "nw must be an even 2^a 3^b size in 16..4096");
  const bool special = !c->fft_generic && fft2_size(nw);  // size-specialised passes, else generic
  if (in->n_interp < 1 || in->n_interp > 3) return fail(CUBE_E_ARG, "n_interp must be 1 (NGP), 2 (CIC) or 3 (TSC)");
  if (in->n_int < 0 || in->n_int > PK_MAX_NINT) return fail(CUBE_E_ARG, "n_int must be in 0..4");
  const int nyq = nw / 2;
  const int64_t nbin = std::lround((float)nyq * std::sqrt(3.f));  // powerspectrum.f90:15
  if (nxi < 10 * (nbin + 1)) return fail(CUBE_E_ARG, "xi needs 10*(nbin+1) floats, nbin = nint(nw/2*sqrt(3))");
  CK(cudaSetDevice(c->device));
  int rc = add_fft(c, nw);
  if (rc) return rc;
  const Geo& G = c->G;
  const bool fixed = c->P.deposit_mode == CUBE_DEPOSIT_FIXED;
  const Pitch pt = pitch_of(c, nw, false);
  const int64_t n3 = (int64_t)nw * nw * nw;
  const size_t mbytes = (mesh_bytes(c, nw, 1, false) + 255) / 256 * 256;
  const size_t abytes = fixed ? (size_t)n3 * 8 : 0;
  // the mesh (and the fixed-point sums) in the arena when they fit, else temporaries
  void* big = nullptr;
  char* base = static_cast<char*>(c->arena);
  if (mbytes + abytes > c->arena_bytes) {
    CK(cudaMalloc(&big, mbytes + abytes));
    base = static_cast<char*>(big);
  }
  float* mesh = reinterpret_cast<float*>(base);
  long long* acc = reinterpret_cast<long long*>(base + mbytes);
  const int nred = 4 * 148;
  const size_t nbins4 = 4 * (size_t)(nbin + 1), nbins3 = 3 * (size_t)(nbin + 1);
  void* small = nullptr;
  const size_t sbytes = (nred + 1 + nbins4 + nbins3) * sizeof(double) + 2 * sizeof(int);
  if (cudaMalloc(&small, sbytes) != cudaSuccess) {
    if (big) cudaFree(big);
    return fail(CUBE_E_CUDA, "cudaMalloc of the power-spectrum sums failed");
  }
  double* partial = static_cast<double*>(small);
  double* total = partial + nred;
  double* bins = total + 1;
  double* cb = bins + nbins4;
  int* mm = reinterpret_cast<int*>(cb + nbins3);
  auto cleanup = [&]() {
    cudaFree(small);
    if (big) cudaFree(big);
  };
#define PK_CK(call)                                                                     \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      cleanup();                                                                        \
      return fail(CUBE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    }                                                                                   \
  } while (0)
  PK_CK(cudaEventRecord(c->ev[0], c->s));
  const int64_t np = c->np;
  // cicpower.f90:76-98
  if (fixed) {
    PK_CK(cudaMemsetAsync(acc, 0, abytes, c->s));
    LAUNCH(c, K_PK_DEP, 1, k_cic_deposit<true><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, acc, nw, nw, (int64_t)nw * nw));
    LAUNCH(c, K_PK_DEP, 1, k_pk_density<true><<<nred, 256, 0, c->s>>>(acc, mesh, nw, pt.pr, pt.plr, partial));
  } else {
    PK_CK(cudaMemsetAsync(mesh, 0, mbytes, c->s));
    LAUNCH(c, K_PK_DEP, 1, k_cic_deposit<false><<<nblk(np), 256, 0, c->s>>>(G, np, c->xp, c->pcell, mesh, nw, pt.pr, pt.plr));
    LAUNCH(c, K_PK_DEP, 1, k_pk_density<false><<<nred, 256, 0, c->s>>>(nullptr, mesh, nw, pt.pr, pt.plr, partial));
  }
  k_pk_sum_partials<<<1, 256, 0, c->s>>>(partial, nred, total);
  double rho8 = 0.0;
  PK_CK(cudaMemcpyAsync(&rho8, total, sizeof(double), cudaMemcpyDeviceToHost, c->s));
  PK_CK(cudaStreamSynchronize(c->s));
  // cicpower.f90:171-180: mean = rho8/nw/nw/nw, delta = rho/mean - 1
  const double mean = rho8 / (double)nw / (double)nw / (double)nw;
  const int mm0[2] = {0x7fffffff, (int)0x80000000};
  PK_CK(cudaMemcpyAsync(mm, mm0, sizeof(mm0), cudaMemcpyHostToDevice, c->s));
  LAUNCH(c, K_PK_DEP, 1, k_pk_delta<<<nred, 256, 0, c->s>>>(mesh, nw, pt.pr, pt.plr, mean, mm));
  if (delta) {
    if (pt.pr == nw)  // plane-compact: each plane's rows are contiguous
      PK_CK(cudaMemcpy2DAsync(delta, (size_t)nw * nw * 4, mesh, pt.psb, (size_t)nw * nw * 4, nw, cudaMemcpyDeviceToHost, c->s));
    else
      PK_CK(cudaMemcpy2DAsync(delta, (size_t)nw * 4, mesh, pt.rp, (size_t)nw * 4, (size_t)nw * nw, cudaMemcpyDeviceToHost, c->s));
  }
  // powerspectrum.f90:148-187
  if (special) fft2_forward_dispatch(c, nw, mesh, pt, K_PK_FFT);
  else fft_forward_generic(c, nw, mesh, pt, K_PK_FFT);
  PK_CK(cudaMemsetAsync(bins, 0, nbins4 * sizeof(double), c->s));
  smem_optin(k_pk_bin, nbins4 * sizeof(double));
  LAUNCH(c, K_PK_BIN, 1, k_pk_bin<<<nred, 256, nbins4 * sizeof(double), c->s>>>(
                             reinterpret_cast<const float2*>(mesh), nw, pt.pc, pt.plc, (int)nbin, (float)np, in->n_interp, bins));
  std::vector<double> hb(nbins4), hc(nbins3);
  int hmm[2];
  PK_CK(cudaMemcpyAsync(hb.data(), bins, nbins4 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
  PK_CK(cudaMemcpyAsync(hmm, mm, sizeof(hmm), cudaMemcpyDeviceToHost, c->s));
  PK_CK(cudaStreamSynchronize(c->s));
  for (int64_t b = 0; b <= nbin; ++b) {
    float* x = xi + 10 * b;
    for (int r = 0; r < 10; ++r) x[r] = 0.f;
    x[0] = (float)hb[4 * b];
    x[1] = (float)hb[4 * b + 1] / x[0];
    x[2] = (float)hb[4 * b + 2] / x[0];
    x[3] = (float)hb[4 * b + 3] / x[0];
    x[4] = x[3];
  }
  // powerspectrum.f90:194-201: up to n_corr pk_correction passes while alpha is a number
  float alpha = 0.f;
  int done = 0;
  const int64_t npairs = (int64_t)(nyq + 1) * (nyq + 2) / 2;
  const size_t smc3 = nbins3 * sizeof(double);
  smem_optin(k_pk_alias<0>, smc3);
  smem_optin(k_pk_alias<1>, smc3);
  smem_optin(k_pk_alias<2>, smc3);
  smem_optin(k_pk_alias<3>, smc3);
  smem_optin(k_pk_alias<4>, smc3);
  for (int it = 0; it < in->n_corr; ++it) {
    if (it > 0 && std::isnan(alpha)) break;
    alpha = (std::log(pk_interp1(xi, nbin, 1, 4, (float)nyq)) - std::log(pk_interp1(xi, nbin, 1, 4, (float)nyq / 2))) /
            std::log(2.f);
    if (std::isnan(alpha)) continue;
    PK_CK(cudaMemsetAsync(cb, 0, nbins3 * sizeof(double), c->s));
    const int p2 = 2 * in->n_interp;
    switch (in->n_int) {
      case 0: LAUNCH(c, K_PK_ALIAS, 1, k_pk_alias<0><<<(unsigned)npairs, 128, smc3, c->s>>>(nw, (int)nbin, alpha, p2, cb)); break;
      case 1: LAUNCH(c, K_PK_ALIAS, 1, k_pk_alias<1><<<(unsigned)npairs, 128, smc3, c->s>>>(nw, (int)nbin, alpha, p2, cb)); break;
      case 2: LAUNCH(c, K_PK_ALIAS, 1, k_pk_alias<2><<<(unsigned)npairs, 128, smc3, c->s>>>(nw, (int)nbin, alpha, p2, cb)); break;
      case 3: LAUNCH(c, K_PK_ALIAS, 1, k_pk_alias<3><<<(unsigned)npairs, 128, smc3, c->s>>>(nw, (int)nbin, alpha, p2, cb)); break;
      default: LAUNCH(c, K_PK_ALIAS, 1, k_pk_alias<4><<<(unsigned)npairs, 128, smc3, c->s>>>(nw, (int)nbin, alpha, p2, cb)); break;
    }
    PK_CK(cudaMemcpyAsync(hc.data(), cb, nbins3 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    PK_CK(cudaStreamSynchronize(c->s));
    for (int64_t b = 1; b <= nbin; ++b) {
      const float ratio = (float)hc[3 * b + 2] / (float)hc[3 * b];
      xi[10 * b + 4] = xi[10 * b + 3] / ratio;
    }
    ++done;
  }
  // powerspectrum.f90:203-206: k in h/Mpc, power in (Mpc/h)^3
  const double PI = 3.141592653589793;
  const float box = c->P.box, box3 = pk_powi(box, 3);
  for (int64_t b = 0; b <= nbin; ++b) {
    float* x = xi + 10 * b;
    x[1] = (float)((double)x[1] * (2 * PI) / (double)box);
    x[2] = x[2] * box3;
    x[3] = x[3] * box3;
    x[4] = x[4] * box3;
  }
  PK_CK(cudaEventRecord(c->ev[1], c->s));
  PK_CK(cudaGetLastError());
  PK_CK(cudaEventSynchronize(c->ev[1]));
  prof_collect(c);
  if (out) {
    memset(out, 0, sizeof(*out));
    out->nbin = nbin;
    out->mean = mean;
    out->alpha = alpha;
    out->n_corr_done = done;
    out->delta_min = pk_key_to_float(hmm[0]);
    out->delta_max = pk_key_to_float(hmm[1]);
    cudaEventElapsedTime(&out->ms, c->ev[0], c->ev[1]);
  }
  cleanup();
#undef PK_CK
  return 0;
}

// =================================================================================
// Differentiable PM step for the adjoint (dpm.cuh; cube_nu_b200/adjoint.py binds it).
// =================================================================================
struct cube_dpm {
  cube_ctx* c = nullptr;  // stream, FFT tables and the Green table (green1)
  int n = 0;
  float mass = 0.f;
  float* mesh = nullptr;  // in-place FFT mesh, layout pitch_of(c, n, false)
  Pitch pt;
  float4* fm = nullptr;   // force mesh, dense n^3
  float4* lam = nullptr;  // adjoint force deposit, dense n^3
};

namespace {

// Force mesh Fm = grad_h Gconv(rho) of the particles at x.
int dpm_force_mesh(cube_dpm* d, const float* x, int64_t np) {
  cube_ctx* c = d->c;
  const int n = d->n;
  CK(cudaMemsetAsync(d->mesh, 0, mesh_bytes(c, n, 1, false), c->s));
  if (np > 0) k_dpm_deposit<<<nblk(np), 256, 0, c->s>>>(n, np, x, d->mass, d->mesh, d->pt.pr, d->pt.plr);
  launch_fft(c, n, 1, d->mesh, false, 1.f, d->mesh, reinterpret_cast<float2*>(d->mesh), c->green1, (float)n, 3, 1);
  const int64_t n3 = (int64_t)n * n * n;
  k_force_pm1<<<nblk(n3), 256, 0, c->s>>>(n, d->mesh, d->pt.pf, d->pt.plf, d->fm);
  c->launches += 7;
  return 0;
}

int dpm_finish(cube_dpm* d) {
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(d->c->s));
  return 0;
}

}  // namespace

extern "C" {

int cube_dpm_create(int n, float soft, float mass, int device, cube_dpm** out) {
  if (!out) return fail(CUBE_E_ARG, "null argument");
  *out = nullptr;
  if (n < 16 || n % 2 || !smooth23(n)) return fail(CUBE_E_ARG, "dpm mesh side must be an even 2^a 3^b size >= 16");
  if (!(soft >= 0.f) || !(mass > 0.f)) return fail(CUBE_E_ARG, "dpm needs soft >= 0 and mass > 0");
  cube_dpm* d = new cube_dpm();
  cube_ctx* c = new cube_ctx();
  d->c = c;
  d->n = n;
  d->mass = mass;
  c->device = device;
  int rc = 0;
  auto bail = [&](int code) {
    cube_dpm_destroy(d);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return bail(fail(CUBE_E_CUDA, "dpm: device or stream setup failed"));
  rc = add_fft(c, n);
  if (!rc) rc = build_green(c, &c->green1, n, soft, 0.f, 1.f);  // Green.f90 without a range cut, gridsize 1
  if (rc) return bail(rc);
  const size_t big = 200 * 1024;
  cudaFuncSetAttribute(k_fft_x_r2c<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(k_fft_z_green, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  d->pt = pitch_of(c, n, false);
  const int64_t n3 = (int64_t)n * n * n;
  if (cudaMalloc(&d->mesh, mesh_bytes(c, n, 1, false)) != cudaSuccess || cudaMalloc(&d->fm, n3 * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&d->lam, n3 * sizeof(float4)) != cudaSuccess)
    return bail(fail(CUBE_E_CUDA, "dpm: out of device memory"));
  if (cudaStreamSynchronize(c->s) != cudaSuccess) return bail(fail(CUBE_E_CUDA, "dpm: setup failed"));
  *out = d;
  return 0;
}

int cube_dpm_destroy(cube_dpm* d) {
  if (!d) return 0;
  if (d->c) {
    cudaSetDevice(d->c->device);
    if (d->c->s) cudaStreamSynchronize(d->c->s);
  }
  if (d->mesh) cudaFree(d->mesh);
  if (d->fm) cudaFree(d->fm);
  if (d->lam) cudaFree(d->lam);
  if (d->c) cube_gpu_destroy(d->c);
  delete d;
  return 0;
}

int cube_dpm_density(cube_dpm* d, const float* x, int64_t np, float* rho) {
  if (!d || !rho || np < 0 || (np > 0 && !x)) return fail(CUBE_E_ARG, "bad dpm density arguments");
  CK(cudaSetDevice(d->c->device));
  const int n = d->n;
  CK(cudaMemsetAsync(rho, 0, (size_t)n * n * n * 4, d->c->s));
  if (np > 0) k_dpm_deposit<<<nblk(np), 256, 0, d->c->s>>>(n, np, x, d->mass, rho, n, (int64_t)n * n);
  ++d->c->launches;
  return dpm_finish(d);
}

int cube_dpm_density_vjp(cube_dpm* d, const float* x, int64_t np, const float* lam, float* gx) {
  if (!d || !lam || !gx || np < 0 || (np > 0 && !x)) return fail(CUBE_E_ARG, "bad dpm density_vjp arguments");
  CK(cudaSetDevice(d->c->device));
  const int n = d->n;
  if (np > 0)
    k_dpm_grad_gather<<<nblk(np), 256, 0, d->c->s>>>(n, np, x, nullptr, nullptr, lam, n, (int64_t)n * n, d->mass, gx);
  ++d->c->launches;
  return dpm_finish(d);
}

int cube_dpm_drift(cube_dpm* d, float* x, const float* v, int64_t np, float D) {
  if (!d || np < 0 || (np > 0 && (!x || !v))) return fail(CUBE_E_ARG, "bad dpm drift arguments");
  CK(cudaSetDevice(d->c->device));
  if (np > 0) k_dpm_drift<<<nblk(3 * np), 256, 0, d->c->s>>>(d->n, 3 * np, x, v, D);
  ++d->c->launches;
  return dpm_finish(d);
}

int cube_dpm_kdk(cube_dpm* d, float* x, float* v, int64_t np, float D, float K) {
  if (!d || np < 0 || (np > 0 && (!x || !v))) return fail(CUBE_E_ARG, "bad dpm kdk arguments");
  CK(cudaSetDevice(d->c->device));
  if (np > 0) k_dpm_drift<<<nblk(3 * np), 256, 0, d->c->s>>>(d->n, 3 * np, x, v, D);
  int rc = dpm_force_mesh(d, x, np);
  if (rc) return rc;
  if (np > 0) k_dpm_kick<<<nblk(np), 256, 0, d->c->s>>>(d->n, np, x, d->fm, K, v);
  d->c->launches += 2;
  return dpm_finish(d);
}

int cube_dpm_force(cube_dpm* d, const float* x, int64_t np, float* f) {
  if (!d || !f || np < 0 || (np > 0 && !x)) return fail(CUBE_E_ARG, "bad dpm force arguments");
  CK(cudaSetDevice(d->c->device));
  int rc = dpm_force_mesh(d, x, np);
  if (rc) return rc;
  CK(cudaMemsetAsync(f, 0, (size_t)np * 12, d->c->s));
  if (np > 0) k_dpm_kick<<<nblk(np), 256, 0, d->c->s>>>(d->n, np, x, d->fm, 1.f, f);
  ++d->c->launches;
  return dpm_finish(d);
}

int cube_dpm_force_vjp(cube_dpm* d, const float* x, int64_t np, const float* u, float* gx) {
  if (!d || !u || !gx || np < 0 || (np > 0 && !x)) return fail(CUBE_E_ARG, "bad dpm force_vjp arguments");
  CK(cudaSetDevice(d->c->device));
  cube_ctx* c = d->c;
  const int n = d->n;
  const int64_t n3 = (int64_t)n * n * n;
  int rc = dpm_force_mesh(d, x, np);  // Fm at these positions
  if (rc) return rc;
  CK(cudaMemsetAsync(d->lam, 0, n3 * sizeof(float4), c->s));
  if (np > 0) k_dpm_deposit_vec<<<nblk(np), 256, 0, c->s>>>(n, np, x, u, d->lam);
  k_dpm_grad_t<<<nblk(n3), 256, 0, c->s>>>(n, d->lam, d->mesh, d->pt.pr, d->pt.plr);
  launch_fft(c, n, 1, d->mesh, false, 1.f, d->mesh, reinterpret_cast<float2*>(d->mesh), c->green1, (float)n, 3, 1);
  if (np > 0)
    k_dpm_grad_gather<<<nblk(np), 256, 0, c->s>>>(n, np, x, u, d->fm, d->mesh, d->pt.pf, d->pt.plf, d->mass, gx);
  c->launches += 8;
  return dpm_finish(d);
}

int cube_dpm_green(cube_dpm* d, float* out, int64_t nout) {
  if (!d || !out) return fail(CUBE_E_ARG, "null argument");
  const int n = d->n;
  const int64_t cnt = (int64_t)n * n * (n / 2 + 1);
  if (nout < cnt) return fail(CUBE_E_ARG, "buffer too small");
  CK(cudaSetDevice(d->c->device));
  CK(cudaMemcpy(out, d->c->green1, cnt * 4, cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
