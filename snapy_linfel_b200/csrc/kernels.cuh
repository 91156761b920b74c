// kernels.cuh — launchers shared between the translation units of libsnapb.
#pragma once

#include <mutex>
#include <utility>
#include <vector>

#include <string>

#include "common.cuh"

namespace snapb {

// Device buffers of one RK stage.  State arrays are caller-owned; the rest
// live in the workspace (see ws_layout in capi.cu).
struct StageBufs {
  const double* dt;  // device scalar
  double* u;         // hydro_u, updated in place
  double* u0;        // hydro_u at stage 0 (interior kept)
  double* w;         // hydro_w, written from u
  double* s;         // scalar_s (nscalar vars) or null
  double* s0;
  double* r;         // scalar_r of the previous stage (mass-correction term)
  double* D;         // [nvar + nscalar][sv] flux-difference sums, then du
  double* RG;        // [sv] hydrostatic correction rho_grav
  double* DD;        // [nvar][sv] diffusion flux differences (undivided)
  double* R;         // [nscalar][sv] scalar mixing ratio of the stage input
  double* M;         // [nvar][sv] implicit mass correction (IDN row used)
  double* vic;       // implicit-solve scratch
  double* vicT;      // per-layer |A| and J blocks (split column sweep), or null
  int stage;
  double wgt0, wgt1, wgt2;
  int write_du;      // 1: finalize writes du into D instead of updating u
  int vic_du_only;   // 1: the implicit solve leaves du in D (no RK update)
};

// Buffers of one RK stage of the FP32 perturbation form: the state is stored
// as FP32 perturbations about the FP64 reference profile rho_bar(x1),
// p_bar(x1): u' = u - (rho_bar, 0, 0, 0, p_bar/(gamma-1)),
// w' = (rho - rho_bar, v1, v2, v3, p - p_bar).
struct StageBufs32 {
  const double* dt;
  float* u;
  float* u0;
  float* w;
  float* s;
  float* s0;
  float* r;
  float* D;    // [nvar + nscalar][sv] flux-difference sums, then du
  float* R;    // [nscalar][sv]
  double* M;   // [sv] implicit mass correction
  double* vic;
  const double* rb;  // [nc1] reference density (cell centres)
  const double* pb;  // [nc1] reference pressure
  double* pf;        // [nc1+1] x1 face reference pressure
  float* offL;       // [nc1+1] left-state reference offset from pf
  float* offR;       // [nc1+1] right-state reference offset from pf
  float* rbar;       // [nc1] FP64 residual of the reference x1 momentum balance
  float* rbf;        // [nc1] float(rho_bar)
  float* pbf;        // [nc1] float(p_bar)
  int stage;
  double wgt0, wgt1, wgt2;
  int write_du;
  int vic_du_only;
};

// ---------------------------------------------------------------------------
// Batched ensembles: many independent blocks of uneven sizes advanced by one
// persistent launch per sweep, each CTA pulling (member, tile) work items from
// a device counter.
// ---------------------------------------------------------------------------

// One ensemble member (FP32 perturbation form), resident in device memory.
// The stage-dependent fields of b (stage, weights) are set by each launch.
struct Member32 {
  Geo g;
  StageBufs32 b;
  int bc[6];
  int x1_cols;           // columns per x1 tile
  int seglen2, nseg2;    // x2 march: faces per segment, segments
  int seglen3, nseg3;    // x3 march
  int vic_cols;          // columns per implicit-column tile
  int pad;
};

// Work items of one persistent launch: item k belongs to member m when
// prefix[m] <= k < prefix[m + 1]; `counter` is zero when the launch starts.
struct WorkQueue {
  const int64_t* prefix;  // [M + 1]
  int M;
  unsigned long long* counter;
};

// Next (member, tile) for the whole CTA; false when the queue is drained.
// Every thread of the CTA must call it.
// (member, tile) of a work item (false past the last item): binary search of
// the per-member prefix table
__device__ __forceinline__ bool queue_find(const WorkQueue& q, int64_t item, int& m,
                                           int64_t& tile) {
  if (item >= q.prefix[q.M]) return false;
  int lo = 0, hi = q.M - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (q.prefix[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  m = lo;
  tile = item - q.prefix[lo];
  return true;
}

__device__ __forceinline__ bool queue_next(const WorkQueue& q, int& m, int64_t& tile) {
  __shared__ unsigned long long s_item;
  __syncthreads();
  if (threadIdx.x == 0) s_item = atomicAdd(q.counter, 1ULL);
  __syncthreads();
  return queue_find(q, (int64_t)s_item, m, tile);
}

// Raise a kernel's dynamic shared-memory limit above the default 48 KB, once
// per (device, kernel): the attribute belongs to the current device's
// context.  The first launch of each kernel on a device should come before
// any stream capture.
template <class K>
inline void raise_smem_limit(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::vector<std::pair<int, const void*>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  const void* f = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> lock(mu);
  for (auto& d : done)
    if (d.first == dev && d.second == f) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  done.emplace_back(dev, f);
}

// Copy member m's descriptor into shared memory, whole CTA, then barrier.  Call
// it right after queue_next (whose leading barrier ends the previous tile).
// Kernels then read the fields as they need them instead of holding the
// ~50-word struct in registers for the whole tile.
// the same copy by one warp (no CTA barrier; the warp's lanes see it after
// __syncwarp, the others after the next CTA barrier)
__device__ __forceinline__ void load_member_warp(Member32& dst, const Member32* mem, int m) {
  const int* src = reinterpret_cast<const int*>(mem + m);
  int* d = reinterpret_cast<int*>(&dst);
  for (int k = threadIdx.x & 31; k < (int)(sizeof(Member32) / sizeof(int)); k += 32) d[k] = src[k];
  __syncwarp();
}
__device__ __forceinline__ void load_member(Member32& dst, const Member32* mem, int m) {
  static_assert(sizeof(Member32) % sizeof(int) == 0, "member descriptor copy");
  const int* src = reinterpret_cast<const int*>(mem + m);
  int* d = reinterpret_cast<int*>(&dst);
  for (int k = threadIdx.x; k < (int)(sizeof(Member32) / sizeof(int)); k += blockDim.x)
    d[k] = src[k];
  __syncthreads();
}

// Persistent grid of a batched launch: as many CTAs as fit on the GPU at once
// (the occupancy calculator's blocks per SM, optionally capped), never more
// than there are work items.
struct PersistGrid {
  int sms;        // multiprocessors
  int cap;        // CTAs per SM cap (0: occupancy only)
  int64_t tiles;  // work items in the queue
};
template <class K>
inline int persistent_grid(K kernel, int block, size_t smem, const PersistGrid& pg) {
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  if (pg.cap > 0 && pg.cap < per) per = pg.cap;
  int64_t g = (int64_t)per * pg.sms;
  if (g > pg.tiles) g = pg.tiles;
  return (int)(g < 1 ? 1 : g);
}

// persistent launchers of the batched FP32 stage
cudaError_t launch_x1_32_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                               int stage, bool last, const PersistGrid& pg, size_t smem, int C,
                               int nc1max, cudaStream_t st);
cudaError_t launch_march32_batch(int axis, const Member32* mem, const Phys& p,
                                 const WorkQueue& q, int stage, bool first, bool last,
                                 const PersistGrid& pg, cudaStream_t st);
cudaError_t launch_vic_column_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                    int stage, const PersistGrid& pg, int block, int variant,
                                    cudaStream_t st);
cudaError_t launch_vic_finish_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                    int stage, const PersistGrid& pg, cudaStream_t st);
cudaError_t launch_vic_cr32_batch(const Member32* mem, const Phys& p, const WorkQueue& q,
                                  int stage, const PersistGrid& pg, int max_layers,
                                  cudaStream_t st);
// the fused implicit-solve kernel (vicf.cu): one launch per solve, tiles of
// vicf_tile_columns() columns
cudaError_t launch_vicf_batch(const Member32* mem, const Phys& p, const WorkQueue& q, int stage,
                              const PersistGrid& pg, cudaStream_t st);
int vicf_tile_columns();
cudaError_t launch_bc32_batch(const Member32* mem, const Phys& p, const WorkQueue& q, int kind,
                              double igm1, const PersistGrid& pg, cudaStream_t st);
size_t x1_smem32_per_column(const Geo& g, int nvt);
int x1_columns_pow2(int c);  // x1 tile width rounded down to a power of two
// shared memory of an x1 tile of C columns in a launch whose longest column is nc1max
size_t x1_smem32_bytes(int nc1max, int nvt, int C);
cudaError_t launch_x1_ghost_revision32_batch(const Member32* mem, const Phys& p,
                                             const WorkQueue& q, const PersistGrid& pg,
                                             cudaStream_t st);
StageBufs32 bufs32_of(const snapb_hydro_config& c, void* ws);
size_t workspace_size_f32_of(const snapb_hydro_config& c);
constexpr int kVicFinishCols = 32;    // columns per implicit-finish tile
// work items of the small batched phases (cells or ghost slots per queue item):
// large enough that the queue fetch and the CTA's reductions are amortised
constexpr int kCflItem = 8192;       // interior cells per CFL item
constexpr int kShellItem = 2048;     // ghost-shell slots per boundary-fill item
constexpr int kRevisionItem = 1024;  // ghost-revision slots per item

// RK3 (Shu-Osher) stage weights: u = wgt0*u0 + wgt1*u + wgt2*du
inline void rk3_weights(int stage, double& a, double& b, double& c) {
  static const double W[3][3] = {{1., 0., 1.}, {3. / 4., 1. / 4., 1. / 4.},
                                 {1. / 3., 2. / 3., 2. / 3.}};
  a = W[stage][0];
  b = W[stage][1];
  c = W[stage][2];
}

// the stage fields of a member's buffers (batched launches set them per stage)
__device__ __forceinline__ void set_stage32(StageBufs32& b, int stage) {
  double w0 = 1., w1 = 0., w2 = 1.;
  if (stage == 1) w0 = 3. / 4., w1 = 1. / 4., w2 = 1. / 4.;
  if (stage == 2) w0 = 1. / 3., w1 = 2. / 3., w2 = 2. / 3.;
  b.stage = stage;
  b.wgt0 = w0;
  b.wgt1 = w1;
  b.wgt2 = w2;
}

// CFL limit of the FP32 form: the signal speeds |v_d| + cs of one cell in
// FP32 (full density and pressure from the FP32 copies of the reference).  A
// thread keeps the largest speed per axis and turns it into dx_d / a_max_d
// (FP64) once: correctly rounded division is monotone, so the minimum over
// cells of dx / a equals dx / (max over cells of a) however the cells are
// split between threads, and the single-domain and batched reductions agree
// to the bit.
__device__ __forceinline__ void cfl32_speeds(const float* w, int64_t sv, int64_t o, float rbf,
                                             float pbf, float gamma, float (&a)[3]) {
  const float rho = rbf + w[IDN * sv + o], pr = pbf + w[IPR * sv + o];
  const float cs = sqrtf(fdiv(gamma * pr, rho));
#pragma unroll
  for (int d = 0; d < 3; ++d) a[d] = fmaxf(a[d], fabsf(w[(IVX + d) * sv + o]) + cs);
}
// dx_d / a_d for the used axes (1.7e308 for the others)
__device__ __forceinline__ void cfl32_limits(const Geo& g, int use1, int use2, int use3,
                                             const float (&a)[3], double& m1, double& m2,
                                             double& m3) {
  m1 = use1 ? g.dx1 / (double)a[0] : 1.7e308;
  m2 = use2 ? g.dx2 / (double)a[1] : 1.7e308;
  m3 = use3 ? g.dx3 / (double)a[2] : 1.7e308;
  m1 = fmin(m1, 1.7e308);  // (a thread without cells: dx / 0)
  m2 = fmin(m2, 1.7e308);
  m3 = fmin(m3, 1.7e308);
}

// launchers (return a cudaError_t of the launch)
cudaError_t launch_x1(const Geo& g, const Phys& p, const StageBufs& b, bool last,
                      cudaStream_t st);
cudaError_t launch_c2p_only(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_march(int axis, const Geo& g, const Phys& p, const StageBufs& b, bool first,
                         bool last, cudaStream_t st);
cudaError_t launch_finalize(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_diffusion(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_vic(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_vic32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st);
size_t vic_scratch_bytes(const Geo& g, const Phys& p);
size_t vic_column_scratch_bytes(const Geo& g, const Phys& p);
size_t vicf_scratch_bytes(const Geo& g, const Phys& p);
cudaError_t launch_vic_column(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_vicf(const Geo& g, const Phys& p, const StageBufs& b, cudaStream_t st);
cudaError_t launch_vicf32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st);
size_t vic_blocks_bytes(const Geo& g, const Phys& p);
int vic_finish_layers32(const Phys& p);  // layers per implicit-finish tile, FP32 form
// implicit solve of the FP32 form by block cyclic reduction (vic_cr.cu): one
// CTA per column, 3x3 blocks, columns of at most 256 layers
bool vic_cr_applies(const Geo& g, const Phys& p);
size_t vic_cr_smem_bytes(int nl);
cudaError_t launch_vic_cr32(const Geo& g, const Phys& p, const StageBufs32& b, cudaStream_t st);

cudaError_t launch_cons2prim(const Geo& g, const Phys& p, const double* u, double* w,
                             cudaStream_t st);
cudaError_t launch_prim2cons(const Geo& g, const Phys& p, const double* w, double* u,
                             cudaStream_t st);
cudaError_t launch_bc(const Geo& g, const snapb_hydro_config& c, double* var, int nv, int kind,
                      cudaStream_t st);
cudaError_t launch_cfl(const Geo& g, const Phys& p, const double* w, double* slots,
                       double* dt_out, cudaStream_t st);
cudaError_t launch_cfl_final(const Geo& g, const Phys& p, unsigned long long* slots,
                             double* dt_out, cudaStream_t st);
cudaError_t launch_scale_dt(const double* dt_in, double cfl, int redo, double* dt_out,
                            cudaStream_t st);
cudaError_t launch_check_positive(const Geo& g, const Phys& p, const double* u, int* flags,
                                  cudaStream_t st);
cudaError_t launch_reconstruct(const Geo& g, const Phys& p, int dim, int group, const double* w,
                               int nv, double* wlr, cudaStream_t st);
cudaError_t launch_riemann(const Geo& g, const Phys& p, int solver, int dim, const double* wl,
                           const double* wr, int nv, double* flx, double* fp, const double* vel,
                           cudaStream_t st);

// CUDA-event pair around a kernel sequence while snapb_timing_enable is on
// (kind: a SNAPB_K_* value); defined in capi.cu
struct ScopedTimer {
  int kind;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  ScopedTimer(int k, cudaStream_t s);
  ~ScopedTimer();
  ScopedTimer(const ScopedTimer&) = delete;
  ScopedTimer& operator=(const ScopedTimer&) = delete;
};

// argument validation and last-error reporting shared with entry points that
// live outside capi.cu
const char* internal_check_config(const snapb_hydro_config* c);
int internal_fail(int code, const std::string& msg);

// bytes of dynamic shared memory the x1 column kernel needs per column
size_t x1_smem_per_column(const Geo& g, int nvt);
int x1_columns_per_cta(const Geo& g, int nvt);

}  // namespace snapb
