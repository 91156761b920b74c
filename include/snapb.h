/*
 * snapb.h — C ABI of the B200 hydro step (snapy finite-volume forward path).
 *
 * Every entry point takes plain device pointers, a pointer to a
 * snapb_hydro_config and a CUDA stream passed as void* (NULL = legacy default
 * stream).  No torch types cross this boundary.  Arrays use snapy's layout
 * [nvar, nc3, nc2, nc1] in row-major order, x1 (vertical) contiguous, with
 * nc = nx + 2*nghost on active axes and nc = 1 on inactive ones
 * (reference: src/hydro/hydro.cpp:87-115, src/coord/coordinate.hpp:58-60).
 * Variable order is IDN=0, IVX=1, IVY=2, IVZ=3, IPR=4 (src/snap.h:34-46).
 *
 * Every function returns SNAPB_OK (0) or a non-zero status; snapb_last_error()
 * gives the message of the last failure on the calling thread.  The caller
 * owns every buffer; scratch memory is sized with snapb_workspace_size().
 * Scalars that change every step (dt) are read from DEVICE memory so that a
 * step can be captured in a CUDA graph and replayed.
 */
#ifndef SNAPB_H
#define SNAPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNAPB_ABI_VERSION 1

/* interpolation types; factory: src/recon/interpolation.cpp:11-39 */
enum {
  SNAPB_RECON_DC = 0,
  SNAPB_RECON_PLM = 1,
  SNAPB_RECON_CP3 = 2,
  SNAPB_RECON_CP5 = 3,
  SNAPB_RECON_WENO3 = 4,
  SNAPB_RECON_WENO5 = 5
};

/* Riemann solvers; factory: src/riemann/riemann_solver.cpp:47-68 */
enum {
  SNAPB_RIEMANN_ROE = 0,
  SNAPB_RIEMANN_LMARS = 1,
  SNAPB_RIEMANN_HLLC = 2,
  SNAPB_RIEMANN_UPWIND = 3
};

/* external boundary functions; registry: src/bc/bc_func.cpp:4-63 */
enum {
  SNAPB_BC_CUSTOM = 0, /* no-op, as custom_inner/custom_outer */
  SNAPB_BC_REFLECTING = 1,
  SNAPB_BC_PERIODIC = 2,
  SNAPB_BC_OUTFLOW = 3
};

/* variable kinds for boundary fills; src/snap.h:53-62 */
enum { SNAPB_PRIMITIVE = 0, SNAPB_CONSERVED = 1, SNAPB_SCALAR = 2 };

/* status codes */
enum {
  SNAPB_OK = 0,
  SNAPB_ERR_ARG = 1,
  SNAPB_ERR_CUDA = 2,
  SNAPB_ERR_UNSUPPORTED = 3,
  SNAPB_ERR_WORKSPACE = 4,
  SNAPB_ERR_TIMEOUT = 5
};

/*
 * One mesh block's hydro configuration.  Mirrors the YAML keys that
 * MeshBlockOptionsImpl::from_yaml reads for this path (geometry.*,
 * dynamics.equation-of-state.*, dynamics.reconstruct.*,
 * dynamics.riemann-solver.type, integration.implicit-scheme,
 * forcing.const-gravity.*, forcing.diffusion.*,
 * boundary-condition.external.*, scalar.nvar).
 */
typedef struct snapb_hydro_config {
  int32_t nx1, nx2, nx3; /* interior cells per axis; 1 = inactive axis */
  int32_t nghost;        /* ghost layers on active axes */
  int32_t nvar;          /* hydro variables (5 for the ideal gas) */
  int32_t nscalar;       /* passive scalars carried in scalar_s */
  double x1min, x1max, x2min, x2max, x3min, x3max;
  double gammad; /* ratio of specific heats */
  double rgas;   /* specific gas constant R = Rgas / weight (W->T) */
  int32_t recon1_type, recon1_shock, recon1_scale;    /* vertical (x1) */
  int32_t recon23_type, recon23_shock, recon23_scale; /* horizontal */
  int32_t scalar_recon_type, scalar_recon_scale;
  int32_t riemann;
  int32_t implicit_scheme; /* 0 none, 1 partial 3x3, 9 full 5x5 */
  double grav1, grav2, grav3, non_hydrostatic;
  double nu_iso, kappa_iso;
  int32_t bc[6]; /* x1-inner, x1-outer, x2-inner, x2-outer, x3-inner, x3-outer */
  int32_t disable_flux[3];
  int32_t reserved;
} snapb_hydro_config;

/* ---- library ---- */
int snapb_abi_version(void);
const char* snapb_last_error(void);

/* Bytes of device scratch that snapb_stage / snapb_hydro_forward need. */
size_t snapb_workspace_size(const snapb_hydro_config* cfg);

/* ---- equation of state (ideal gas) ---- */

/* U -> W over the whole array, ghosts included.
 * Replaces IdealGasImpl::_cons2prim (src/eos/ideal_gas.cpp:90-109) and the
 * ideal_gas_cons2prim DispatchStub (src/eos/eos_dispatch.cu:16-30). */
int snapb_cons2prim(const snapb_hydro_config* cfg, const double* u, double* w,
                    void* stream);

/* W -> U over the whole array.
 * Replaces IdealGasImpl::_prim2cons (src/eos/ideal_gas.cpp:67-88). */
int snapb_prim2cons(const snapb_hydro_config* cfg, const double* w, double* u,
                    void* stream);

/* ---- operator level (one module call each) ---- */

/* wlr[2, nv, nc3, nc2, nc1] = reconstruction of w along dim (3 = x1, 2 = x2,
 * 1 = x3).  group 0 = hydro variables with the vertical (dim 3) or horizontal
 * (dim 1, 2) options; group 1 = passive scalars (interp1 for every variable,
 * then clamp at 0).  Replaces ReconstructImpl::forward
 * (src/recon/reconstruct.cpp:75-154) with the call_weno5 / call_poly5 /
 * PLM stubs it dispatches to (src/recon/recon_dispatch.hpp:9-18). */
int snapb_reconstruct(const snapb_hydro_config* cfg, int dim, int group,
                      const double* w, int nv, double* wlr, void* stream);

/* flx[nv, ...] (and face_pressure[nc3, nc2, nc1] when not NULL) from the
 * left/right states along dim.  solver = SNAPB_RIEMANN_*; for UPWIND `vel`
 * is the face velocity (mass flux) array.  Replaces
 * RiemannSolverImpl::forward and the call_hllc / call_lmars / call_roe stubs
 * (src/riemann/riemann_dispatch.hpp:10-20, src/riemann/hllc.cpp:30-106,
 * src/riemann/lmars.cpp:30-103, src/riemann/roe.cpp:14-59,
 * src/riemann/riemann_solver.cpp:544-553). */
int snapb_riemann(const snapb_hydro_config* cfg, int solver, int dim,
                  const double* wl, const double* wr, int nv, double* flx,
                  double* face_pressure, const double* vel, void* stream);

/* ---- block level ---- */

/* Stage tendency du (already multiplied by dt) of the hydro forward step:
 * cons2prim into w, hydrostatic x1 ghost revision, fused per-direction
 * reconstruct + Riemann + flux difference, gravity, hydrostatic correction
 * and the vertically implicit correction.  mass_corr (may be NULL when the
 * implicit scheme is off) receives the implicit mass fix per cell.
 * Replaces HydroImpl::forward (src/hydro/hydro_forward.cpp:14-217). */
int snapb_hydro_forward(const snapb_hydro_config* cfg, const double* dt,
                        const double* u, double* w, double* du,
                        double* mass_corr, void* workspace,
                        size_t workspace_bytes, void* stream);

/* Vertically implicit correction of a stage tendency, in place.  du holds
 * -dt*div + forcing on interior cells; on return its interior carries the
 * VIC result (block-tridiagonal solve per x1 column, 3x3 for scheme 1, 5x5
 * for scheme 9, then the MS-VIC mass redistribution).  w must hold the
 * primitive state including the x1 ghost cells.  mass_corr (NULL allowed,
 * [nvar, nc3, nc2, nc1]) receives the mass fix in its IDN row at interior
 * cells; other entries are left untouched.  The workspace must hold
 * snapb_workspace_size(cfg) bytes.  Replaces ImplicitHydroImpl::forward
 * (src/implicit/implicit_hydro.cpp:99-189), which returns du_new - du_old
 * instead of updating du. */
int snapb_implicit_correction(const snapb_hydro_config* cfg, const double* dt,
                              double* du, const double* w, double* mass_corr,
                              void* workspace, size_t workspace_bytes,
                              void* stream);

/* The same correction as snapb_implicit_correction, for callers that cannot
 * allocate device memory when they run it (inside a CUDA-graph capture, on a
 * host whose device memory is pre-partitioned, or from a language binding
 * without an allocator).  No reference counterpart: snapy always allocates
 * its implicit-solve buffers.  It allocates nothing and takes no workspace:
 * the column-solve scratch is a fixed 32 MiB array in the library's device
 * memory, present on every GPU that loads the library until the process
 * exits, so problems needing more (nx1 * columns * (N*N+N) * 8 bytes, N = 3
 * or 5) are rejected with SNAPB_ERR_ARG.  The first call on a device looks up
 * that array's address (once per device), so make it before any stream
 * capture.  The looked-up address is kept for the life of the process: after
 * cudaDeviceReset (or any teardown of the device's primary context) in the
 * same process it is stale, so do not call this entry point again after such
 * a reset.  All calls share the one array: calls whose kernels overlap on the
 * GPU (different streams, or different host threads) race on it; serialize
 * them.  The solve writes every scratch entry before reading it, so nothing
 * is carried over from the previous call. */
int snapb_implicit_correction_noalloc(const snapb_hydro_config* cfg,
                                      const double* dt, double* du,
                                      const double* w, double* mass_corr,
                                      void* stream);

/* One RK stage of a mesh block, in place: du = forward(u), optional scalar
 * transport, u = wght0*u0 + wght1*u + wght2*du, boundary fills.  At stage 0
 * u0 (and s0) are filled from u (and s).  s, s0, r may be NULL when
 * cfg->nscalar == 0.  Replaces MeshBlockImpl::advance_local
 * (src/mesh/meshblock.cpp:577-786) with its harp RK3 combination
 * (stage weights (1,0,1), (3/4,1/4,1/4), (1/3,2/3,2/3)). */
int snapb_stage(const snapb_hydro_config* cfg, int stage, const double* dt,
                double* u, double* u0, double* w, double* s, double* s0,
                double* r, void* workspace, size_t workspace_bytes,
                void* stream);

/* External boundary fills of var[nv, nc3, nc2, nc1] in the order x1-inner,
 * x1-outer, x2-inner, x2-outer, x3-inner, x3-outer; kind = SNAPB_PRIMITIVE,
 * SNAPB_CONSERVED or SNAPB_SCALAR.  Replaces the bfuncs loop
 * (src/mesh/meshblock.cpp:717-730) over src/bc/bc_func.cpp:7-63. */
int snapb_bc_apply(const snapb_hydro_config* cfg, double* var, int nv,
                   int kind, void* stream);

/* Hyperbolic (and diffusive) time-step limit from w, written to *dt_out
 * (device).  The CFL factor and redo halving are NOT applied.
 * Replaces HydroImpl::max_time_step (src/hydro/hydro.cpp:118-180) and
 * DiffusionImpl::max_time_step (src/forcing/diffusion.cpp:242-265). */
int snapb_max_time_step(const snapb_hydro_config* cfg, const double* w,
                        double* dt_out, void* workspace,
                        size_t workspace_bytes, void* stream);

/* dt_out = cfl * 2^-redo * (*dt_in) on the device. */
int snapb_scale_dt(const double* dt_in, double cfl, int redo, double* dt_out,
                   void* stream);

/* Positivity screen of the interior (device ints): flags[0] = 1 if some
 * density <= 0, flags[1] = 1 if some total energy <= 0, flags[2] = 1 if some
 * cons2prim pressure <= 0.  A step is redone when flags[0] || (flags[1] &&
 * flags[2]), as MeshBlockImpl::check_redo decides
 * (src/mesh/meshblock.cpp:974-1016). */
int snapb_check_positive(const snapb_hydro_config* cfg, const double* u,
                         int* flags, void* stream);

/* ---- slab domain decomposition: ghost-zone messages ----
 * A slab is `width` consecutive indices along x2 (axis 2) or x3 (axis 3) of
 * var[nv, nc3, nc2, nc1], from `start`, with the full extent of the other
 * axes.  snapb_pack_slab copies it into buf in the row-major order of
 * var[:, slab] ([nv][nc3][width][nc1] or [nv][width][nc2][nc1]);
 * snapb_unpack_slab writes such a buffer into a slab.  The exchange of a
 * decomposed block packs the ng interior layers next to each internal face
 * into a send buffer in the sender's memory, moves it as one message and
 * unpacks it into the receiver's ghost layers.  Replaces the face copies of
 * LayoutImpl's exchange (src/layout/layout.cpp:361-634). */
int snapb_pack_slab(const snapb_hydro_config* cfg, int axis, int start,
                    int width, const double* var, int nv, double* buf,
                    void* stream);
int snapb_unpack_slab(const snapb_hydro_config* cfg, int axis, int start,
                      int width, double* var, int nv, const double* buf,
                      void* stream);

/* ---- FP32 perturbation form ----
 * The state is stored in FP32 as perturbations about an FP64 reference
 * profile rho_bar(x1), p_bar(x1) (x1 = vertical, [nc1] device arrays, ghosts
 * included): u' = u - (rho_bar, 0, 0, 0, p_bar/(gamma-1)) and
 * w' = (rho - rho_bar, v1, v2, v3, p - p_bar).  The sweeps run in FP32; the
 * reference's own x1 pressure-gradient / gravity balance, the isentropic
 * ghost revision and the implicit elimination run in FP64, and the momentum
 * fluxes carry pressure relative to an FP64 face reference, so the
 * hydrostatic pressure never enters an FP32 difference.  No reference
 * counterpart: snapy computes in FP64 (or plain FP32) throughout.
 * Requirements: active x1, non-hydrostatic = 1, no diffusion, and a linear x1
 * pressure interpolation (cp5/cp3/dc — WENO5 with shock: false) whenever a
 * reference pressure is given.  Call snapb_reference_f32 once per reference
 * (it fills tables in the workspace) before the other calls. */
size_t snapb_workspace_size_f32(const snapb_hydro_config* cfg);
int snapb_reference_f32(const snapb_hydro_config* cfg, const double* ref_rho,
                        const double* ref_p, void* workspace,
                        size_t workspace_bytes, void* stream);
/* kind = SNAPB_CONSERVED (u <-> u') or SNAPB_PRIMITIVE (w <-> w') */
int snapb_to_perturbation(const snapb_hydro_config* cfg, int kind,
                          const double* in, float* out, void* workspace,
                          size_t workspace_bytes, void* stream);
int snapb_from_perturbation(const snapb_hydro_config* cfg, int kind,
                            const float* in, double* out, void* workspace,
                            size_t workspace_bytes, void* stream);
int snapb_stage_f32(const snapb_hydro_config* cfg, int stage, const double* dt,
                    float* u, float* u0, float* w, float* s, float* s0,
                    float* r, void* workspace, size_t workspace_bytes,
                    void* stream);
int snapb_bc_apply_f32(const snapb_hydro_config* cfg, float* var, int nv,
                       int kind, void* workspace, size_t workspace_bytes,
                       void* stream);
int snapb_max_time_step_f32(const snapb_hydro_config* cfg, const float* w,
                            double* dt_out, void* workspace,
                            size_t workspace_bytes, void* stream);

/* ---- batched ensembles (FP32 perturbation form) ----
 * No counterpart in the reference, which advances one MeshBlock per call:
 * many independent blocks of uneven sizes (same physics, same active axes)
 * advance together.  Each sweep of a stage is one persistent launch over all
 * members whose CTAs pull (member, tile) work items from a device counter.
 * Each member's state is the FP32 perturbation form of snapb_stage_f32, with
 * its own FP32 workspace on which snapb_reference_f32 has run.  The plan
 * (host object) is created once, then bound to a device workspace of
 * snapb_ensemble_workspace_size bytes; every call is stream ordered and
 * graph-capturable (dt per member stays on the device).  Diffusion and
 * non_hydrostatic < 1 are not batched. */
typedef struct snapb_member_f32 {
  snapb_hydro_config cfg;
  float *u, *u0, *w, *s, *s0, *r; /* as snapb_stage_f32 */
  void* workspace;                /* the member's FP32 workspace */
  size_t workspace_bytes;
} snapb_member_f32;

/* tile shapes and kernel variants; 0 = default.  x1_columns: columns per x1
 * tile (a power of two); march_segment: faces per x2/x3 segment; ctas_per_sm:
 * persistent CTAs per SM cap; vic_kernel: the implicit solve (0 the column
 * kernel + finish kernel; 1 block cyclic reduction, one CTA per column, where
 * it applies: 3x3 blocks and columns of at most 256 layers, else 0; 2 the
 * fused kernel: blocks, twisted elimination from both column ends, back
 * substitution and finish in one launch); vic_block: columns per tile of the
 * column kernel (32, 64 or 128); vic_regs: its register budget (0 the
 * compiler's, 1 ~168, 2 128). */
typedef struct snapb_ensemble_tuning {
  int32_t x1_columns, march_segment, ctas_per_sm, vic_block, vic_regs, vic_kernel;
} snapb_ensemble_tuning;

typedef struct snapb_ensemble snapb_ensemble; /* opaque host-side plan */

int snapb_ensemble_create(const snapb_member_f32* members, int n,
                          const snapb_ensemble_tuning* tune, snapb_ensemble** out);
size_t snapb_ensemble_workspace_size(const snapb_ensemble* e);
/* copies the member descriptors and work-queue tables into the workspace */
int snapb_ensemble_bind(snapb_ensemble* e, void* workspace, size_t workspace_bytes,
                        void* stream);
/* re-plans with new tile shapes (within the bound workspace) and re-uploads */
int snapb_ensemble_set_tuning(snapb_ensemble* e, const snapb_ensemble_tuning* tune,
                              void* stream);
/* device array [n]: the members' dt, written by snapb_ensemble_max_time_step_f32
 * (or by the caller) and read by every stage */
const double* snapb_ensemble_dt(const snapb_ensemble* e);
/* dt_m = factor * CFL limit of member m's w (factor = cfl * 2^-redo) */
int snapb_ensemble_max_time_step_f32(snapb_ensemble* e, double factor, void* stream);
/* one RK stage of every member: x1, x2, x3 sweeps, implicit solve, boundary
 * fills, each one persistent launch */
int snapb_ensemble_stage_f32(snapb_ensemble* e, int stage, void* stream);
void snapb_ensemble_destroy(snapb_ensemble* e);

/* ---- adjoint (reverse mode) of the FP64 stage ----
 * No counterpart in the reference, which has no adjoint: these are the
 * `*_adjoint` entry points of the hydro step.  dt is a constant of the
 * adjoint (the CFL choice is not differentiated); every switch of the
 * forward path (Riemann wave selections, upwinding, clamps) is differentiated
 * on the branch the forward pass takes at the given state.  Supported: all
 * reconstructions and hydro Riemann solvers, gravity with non_hydrostatic
 * = 1, implicit schemes 0 / 1 / 9, passive scalars, reflecting / periodic /
 * outflow boundaries; diffusion is rejected with SNAPB_ERR_ARG.
 *
 * The workspace is separate from (and larger than) the forward one. */
size_t snapb_adjoint_workspace_size(const snapb_hydro_config* cfg);

/* Reverse of snapb_stage: u, s are the stage-START state (ghosts filled, as
 * snapb_stage received them); gu_out, gs_out the cotangents of the stage's
 * output (full arrays, after its boundary fill).  Writes gu, gs (full arrays,
 * ghost entries included: cotangents of the input arrays, the wgt1 term of
 * the RK combination included) and ADDS wgt0 * BC^T(gu_out) to gu0, gs0 on
 * the interior (the step-start state; at stage 0 u0 is u, so the caller adds
 * gu0 to gu after the stage-0 reverse).  gs_out, gs, gs0 may be null when
 * nscalar = 0.  The scalar mass-fix term uses s / rho of the stage input as
 * the mixing ratio, which equals the forward's scalar_r after any stage. */
int snapb_stage_adjoint(const snapb_hydro_config* cfg, int stage, const double* dt,
                        const double* u, const double* s, const double* gu_out,
                        const double* gs_out, double* gu, double* gs, double* gu0,
                        double* gs0, void* workspace, size_t workspace_bytes,
                        void* stream);

/* Reverse of snapb_hydro_forward (du including the implicit correction):
 * g_u = (d du / d u)^T g_du over the full array; g_du is read on the
 * interior. */
int snapb_hydro_forward_adjoint(const snapb_hydro_config* cfg, const double* dt,
                                const double* u, const double* g_du, double* g_u,
                                void* workspace, size_t workspace_bytes, void* stream);

/* Reverse of snapb_riemann for the hydro solvers (nv = 5): given the
 * cotangent g_flx of the fluxes at every face, writes g_wl = (dF/dwl)^T g_flx
 * and g_wr = (dF/dwr)^T g_flx (all [5, nc3, nc2, nc1]). */
int snapb_riemann_adjoint(const snapb_hydro_config* cfg, int solver, int dim,
                          const double* wl, const double* wr, const double* g_flx,
                          double* g_wl, double* g_wr, void* stream);

/* Reverse of snapb_bc_apply (out of place): interior cells gather the
 * cotangents of their ghost images (sign flips of reflecting normals for
 * kind != SNAPB_SCALAR), ghost entries of g_out are zero. */
int snapb_bc_adjoint(const snapb_hydro_config* cfg, const double* g_in, double* g_out, int nv,
                     int kind, void* stream);

/* ---- conserved totals (compensated) ----
 * out[v] = cell volume * sum over interior cells of var[v], v < nv, written
 * to DEVICE memory.  Replaces the torch sum of hydro_u * cell_volume over the
 * interior that MeshBlockImpl reports as "mass0"
 * (src/mesh/meshblock.cpp:855-870).  Accumulated as double-double sums in
 * an order fixed by the configuration: the exact total rounded once (to
 * ~2^-100 of the largest partial sum), bit-identical across calls.
 * snapb_conserved_totals_f32 takes the FP32 perturbation form's conserved
 * u' and adds the FP64 reference of the workspace (snapb_reference_f32)
 * back cell by cell, so its totals are of the full state; nv <= nvar.
 * scratch: snapb_totals_scratch_size(cfg, nv) bytes of device memory. */
size_t snapb_totals_scratch_size(const snapb_hydro_config* cfg, int nv);
int snapb_conserved_totals(const snapb_hydro_config* cfg, const double* var, int nv,
                           double* out, void* scratch, size_t scratch_bytes, void* stream);
int snapb_conserved_totals_f32(const snapb_hydro_config* cfg, const float* u, int nv,
                               double* out, const void* workspace, size_t workspace_bytes,
                               void* scratch, size_t scratch_bytes, void* stream);

/* ---- diagnostics: per-kernel device time ----
 * While enabled, snapb_stage, snapb_hydro_forward, snapb_stage_f32 and the
 * adjoint entry points record a CUDA event pair around every kernel (or
 * kernel group) they launch.  snapb_timing_query synchronizes those
 * events and returns the summed device milliseconds and the launch count of
 * one kernel kind.  Enabling clears the record.  (Plays the role of the
 * reference's verbose phase timers, src/hydro/hydro_forward.cpp:26-31.) */
enum {
  SNAPB_K_X1 = 0,   /* U->W + x1 sweep */
  SNAPB_K_DIFF = 1, /* diffusion fluxes */
  SNAPB_K_X2 = 2,   /* x2 sweep */
  SNAPB_K_X3 = 3,   /* x3 sweep */
  SNAPB_K_FINAL = 4,
  SNAPB_K_VIC = 5,  /* implicit column solve */
  SNAPB_K_BC = 6,   /* boundary fills */
  SNAPB_K_ADJ_COMBINE = 7,   /* adjoint: BC^T and RK weights */
  SNAPB_K_ADJ_RECOMPUTE = 8, /* adjoint: forward recompute of w, r, du */
  SNAPB_K_ADJ_VIC = 9,       /* adjoint: implicit solve reverse */
  SNAPB_K_ADJ_X23 = 10,      /* adjoint: x2 / x3 face reverses */
  SNAPB_K_ADJ_X1 = 11,       /* adjoint: x1 faces, gravity, U->W reverse */
  SNAPB_K_COUNT = 12
};
int snapb_timing_enable(int on);
int snapb_timing_query(int kernel, double* total_ms, int* launches);

/* Bulk (TMA-engine) copies: the sweeps that stage their tiles with
 * cp.async.bulk wait on them with a bounded poll; a CTA whose copy did not
 * complete in time gives up its tile and raises a device flag.  Returns the
 * flag (0: every copy completed since the last call; 1: at least one timed
 * out, so the results of those launches are not to be used) and clears it;
 * synchronizes the device; -1 on a CUDA error. */
int snapb_bulk_copy_timeouts(void);

#ifdef __cplusplus
}
#endif

#endif /* SNAPB_H */
