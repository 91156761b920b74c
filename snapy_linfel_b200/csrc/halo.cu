// halo.cu — packing and unpacking of the ghost-zone slabs that the slab
// domain decomposition exchanges between ranks.
//
// A slab is `width` consecutive x2 (axis 2) or x3 (axis 3) indices of an
// array var[nv, nc3, nc2, nc1] starting at `start`, with the full extent of
// the other axes (ghosts included).  Packing writes it into a contiguous
// buffer in the row-major order of var[:, slab] — [nv][nc3][width][nc1] for
// axis 2, [nv][width][nc2][nc1] for axis 3 — which is what a message carries;
// unpacking writes such a buffer back into a slab.  One thread per value,
// consecutive threads along x1, so both sides are coalesced.
//
// Replaces the per-message send/receive buffer handling of LayoutImpl's
// exchange (src/layout/layout.cpp:361-634), which packs the face slices of
// each variable with tensor copies.
#include "kernels.cuh"

namespace snapb {

namespace {

struct Slab {
  int64_t sv, s3, s2;  // strides of var (x1 stride 1)
  int nc1, nk, nj;     // extents of the slab along x1, x3, x2
  int64_t base;        // offset of the slab's first value in var
  int64_t n;           // values per variable
};

Slab make_slab(const Geo& g, int axis, int start, int width) {
  Slab s;
  s.sv = g.sv;
  s.s3 = g.s3;
  s.s2 = g.s2;
  s.nc1 = g.nc1;
  s.nk = axis == 3 ? width : g.nc3;
  s.nj = axis == 2 ? width : g.nc2;
  s.base = axis == 2 ? (int64_t)start * g.s2 : (int64_t)start * g.s3;
  s.n = (int64_t)s.nk * s.nj * s.nc1;
  return s;
}

template <bool PACK>
__global__ void k_slab(Slab s, int nv, double* var, double* buf) {
  const int64_t total = s.n * nv;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = t / s.n;
    int64_t r = t - v * s.n;
    const int i = (int)(r % s.nc1);
    r /= s.nc1;
    const int j = (int)(r % s.nj);
    const int k = (int)(r / s.nj);
    const int64_t o = v * s.sv + s.base + (int64_t)k * s.s3 + (int64_t)j * s.s2 + i;
    if (PACK)
      buf[t] = var[o];
    else
      var[o] = buf[t];
  }
}

const char* check_slab(const snapb_hydro_config* cfg, int axis, int start, int width, int nv) {
  if (const char* e = internal_check_config(cfg)) return e;
  if (axis != 2 && axis != 3) return "axis must be 2 or 3";
  if (nv < 1) return "nv must be >= 1";
  const int nc = axis == 2 ? (cfg->nx2 > 1 ? cfg->nx2 + 2 * cfg->nghost : 1)
                           : (cfg->nx3 > 1 ? cfg->nx3 + 2 * cfg->nghost : 1);
  if (width < 1 || start < 0 || start + width > nc) return "slab outside the array";
  return nullptr;
}

int slab_call(bool pack, const snapb_hydro_config* cfg, int axis, int start, int width,
              double* var, int nv, double* buf, void* stream) {
  const char* who = pack ? "pack_slab" : "unpack_slab";
  if (const char* e = check_slab(cfg, axis, start, width, nv))
    return internal_fail(SNAPB_ERR_ARG, std::string(who) + ": " + e);
  if (!var || !buf) return internal_fail(SNAPB_ERR_ARG, std::string(who) + ": null pointer");
  const Slab s = make_slab(make_geo(*cfg), axis, start, width);
  const int64_t total = s.n * nv;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (pack)
    k_slab<true><<<blocks, 256, 0, st>>>(s, nv, var, buf);
  else
    k_slab<false><<<blocks, 256, 0, st>>>(s, nv, var, buf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return internal_fail(SNAPB_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
  return SNAPB_OK;
}

}  // namespace
}  // namespace snapb

extern "C" {

int snapb_pack_slab(const snapb_hydro_config* cfg, int axis, int start, int width,
                    const double* var, int nv, double* buf, void* stream) {
  return snapb::slab_call(true, cfg, axis, start, width, const_cast<double*>(var), nv, buf,
                          stream);
}

int snapb_unpack_slab(const snapb_hydro_config* cfg, int axis, int start, int width,
                      double* var, int nv, const double* buf, void* stream) {
  return snapb::slab_call(false, cfg, axis, start, width, var, nv, const_cast<double*>(buf),
                          stream);
}

}  // extern "C"
