// Host side of the immersed boundary, shared by the single-block and the
// batched contexts: one body's surface (IBMNodes, variables.h:91-118) and one
// block's interpolation list of that body (IBMList / IBMInfo,
// variables.h:50-89) as device arrays, built from the reference's host
// structures (ibm_search_advanced hands the list over; ibm_iso.c:87).
#pragma once
#include <cuda_runtime.h>

#include <unordered_map>
#include <vector>

#include "../../include/chimera_b200.h"
#include "cb_common.cuh"
#include "cb_ibm.cuh"

namespace cb {

// One immersed body: its surface (IBMNodes) and interpolation list (IBMList)
// in device memory.
struct IbmBody {
  int n_v = 0, n_elmt = 0, n = 0;
  void *surf = nullptr;  // nf (3 per element), u, uold (3 per vertex), tri (3 per element)
  void *list = nullptr;  // node, donors, weights, sweep output
  double *nf = nullptr, *u = nullptr, *uold = nullptr;
  int *tri = nullptr;
  int4 *node = nullptr;
  long long *don = nullptr;
  double *w = nullptr, *out = nullptr, *ustar = nullptr;
  unsigned char *last = nullptr;          // -isothermal 2: the entry that writes its node
  double *iso = nullptr, *pa = nullptr;   // -isothermal 2: per-entry terms, the chain's carried pressure
  IbmDev dev() const {
    IbmDev d;
    d.n = n; d.node = node; d.don = don; d.w = w; d.tri = tri; d.nf = nf; d.u = u; d.uold = uold; d.out = out;
    d.ustar = ustar; d.last = last; d.iso = iso; d.pa = pa;
    return d;
  }
};

static inline void ibm_drop_list(IbmBody &b) {
  if (b.list) cudaFree(b.list);
  b.list = nullptr;
  b.node = nullptr; b.don = nullptr; b.w = nullptr; b.out = nullptr; b.ustar = nullptr;
  b.last = nullptr; b.iso = nullptr; b.pa = nullptr;
  b.n = 0;
}

// A body's list in host form, validated against one block.
struct IbmHostList {
  std::vector<int4> node;
  std::vector<long long> don;
  std::vector<double> w;
  std::vector<unsigned char> lastf;  // -isothermal 2 only
  bool iso2 = false;
  int n() const { return (int)node.size(); }
};

// Validates the n entries of `list` against block `dc` (interface nodes in the
// block, donors in its ghosted box where a direction is periodic, elements of
// a surface of n_elmt) and builds the device layout.  A node listed twice
// keeps its last entry; with -isothermal 2 every entry is kept (the chain of
// Pa walks them all) and `lastf` marks the one that writes its node.
// Returns CB_OK, or CB_E_ARG with *err set.
static inline int ibm_build_list(const DevCfg &dc, bool iso2, int n_elmt, int n, const cb_ibm_info *list,
                                 const double *coor, IbmHostList &h, const char **err) {
  const int m[3] = {dc.mx, dc.my, dc.mz};
  const bool per[3] = {dc.bctype[0] == 7, dc.bctype[2] == 7, dc.bctype[4] == 7};
  std::unordered_map<long long, int> last;
  for (int t = 0; t < n; t++) {
    const cb_ibm_info &f = list[t];
    const int nd[3] = {f.ni, f.nj, f.nk};
    for (int d = 0; d < 3; d++)
      if (nd[d] < 0 || nd[d] >= m[d]) { *err = "interface node outside the block"; return CB_E_ARG; }
    const int dn[9] = {f.i1, f.j1, f.k1, f.i2, f.j2, f.k2, f.i3, f.j3, f.k3};
    for (int a = 0; a < 9; a++) {
      const int d = a % 3, lo = per[d] ? -2 : 0, hi = per[d] ? m[d] + 1 : m[d] - 1;
      if (dn[a] < lo || dn[a] > hi) { *err = "donor node outside the ghosted block"; return CB_E_ARG; }
    }
    if (f.cell < -1 || f.cell >= n_elmt) { *err = "surface element index out of range"; return CB_E_ARG; }
    last[((long long)f.nk * m[1] + f.nj) * m[0] + f.ni] = t;
  }
  std::vector<int> keep;
  keep.reserve(iso2 ? n : last.size());
  h = IbmHostList();
  h.iso2 = iso2;
  for (int t = 0; t < n; t++) {
    const cb_ibm_info &f = list[t];
    const bool is_last = last[((long long)f.nk * m[1] + f.nj) * m[0] + f.ni] == t;
    if (iso2) h.lastf.push_back(is_last ? 1 : 0);
    if (iso2 || is_last) keep.push_back(t);
  }
  const int nk = (int)keep.size();
  h.node.resize(nk);
  h.don.resize(3 * (size_t)nk);
  h.w.resize((size_t)IBM_NW * nk);
  for (int t = 0; t < nk; t++) {
    const cb_ibm_info &f = list[keep[t]];
    h.node[t] = make_int4(f.ni, f.nj, f.nk, f.cell);
    h.don[3 * (size_t)t] = gidx(dc, f.i1, f.j1, f.k1);
    h.don[3 * (size_t)t + 1] = gidx(dc, f.i2, f.j2, f.k2);
    h.don[3 * (size_t)t + 2] = gidx(dc, f.i3, f.j3, f.k3);
    const double *x = coor + 3 * (((size_t)f.nk * m[1] + f.nj) * m[0] + f.ni);
    const double v[IBM_NW] = {f.cr1, f.cr2, f.cr3, f.cs1, f.cs2, f.cs3, f.d_s, f.d_s + f.d_i,
                              x[0] - f.pmin[0], x[1] - f.pmin[1], x[2] - f.pmin[2]};  // ibm_iso.c:2653, 2662-2664
    for (int a = 0; a < IBM_NW; a++) h.w[(size_t)a * nk + t] = v[a];
  }
  return CB_OK;
}

// Device arrays of a built list into b (whose previous list was dropped),
// stream-ordered on st and synchronised.
static inline cudaError_t ibm_list_to_device(IbmBody &b, const IbmHostList &h, cudaStream_t st) {
  const int nk = h.n();
  const bool iso2 = h.iso2;
  const size_t iso_d = iso2 ? (size_t)IBM_ISO_NS * nk + 1 : 0;  // terms, then the carried pressure
  const size_t bytes = sizeof(int4) * nk + sizeof(long long) * 3 * nk +
                       sizeof(double) * ((IBM_NW + 7) * (size_t)nk + iso_d) + (iso2 ? (size_t)nk : 0);
  cudaError_t e = cudaMalloc(&b.list, bytes);
  if (e != cudaSuccess) return e;
  b.node = (int4 *)b.list;
  b.don = (long long *)(b.node + nk);
  b.w = (double *)(b.don + 3 * (size_t)nk);
  b.out = b.w + (size_t)IBM_NW * nk;
  b.ustar = b.out + (size_t)6 * nk;
  if (iso2) {
    b.iso = b.ustar + nk;
    b.pa = b.iso + (size_t)IBM_ISO_NS * nk;
    b.last = (unsigned char *)(b.pa + 1);
    e = cudaMemcpyAsync(b.last, h.lastf.data(), (size_t)nk, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
  }
  b.n = nk;
  if ((e = cudaMemsetAsync(b.ustar, 0, sizeof(double) * nk, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(b.node, h.node.data(), sizeof(int4) * nk, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(b.don, h.don.data(), sizeof(long long) * h.don.size(), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(b.w, h.w.data(), sizeof(double) * h.w.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return e;
  return cudaStreamSynchronize(st);
}

// The surface of a body (triangles nv1..nv3 over n_v vertices, element
// normals) into device memory; vertex velocities start at zero (ibm_read_ucd,
// ibm_io.c:1643-1653).  The caller has dropped the body's list and surface.
// Returns CB_OK, CB_E_ARG with *err set, or CB_E_CUDA.
static inline int ibm_surface_to_device(IbmBody &b, int n_v, int n_elmt, const int *nv1, const int *nv2,
                                        const int *nv3, const double *nf_x, const double *nf_y, const double *nf_z,
                                        cudaStream_t st, const char **err) {
  std::vector<int> tri(3 * (size_t)n_elmt);
  std::vector<double> h(3 * (size_t)n_elmt + 6 * (size_t)n_v, 0.0);
  for (int t = 0; t < n_elmt; t++) {
    const int v[3] = {nv1[t], nv2[t], nv3[t]};
    for (int a = 0; a < 3; a++) {
      if (v[a] < 0 || v[a] >= n_v) { *err = "element vertex index out of range"; return CB_E_ARG; }
      tri[3 * (size_t)t + a] = v[a];
    }
    h[3 * (size_t)t] = nf_x[t]; h[3 * (size_t)t + 1] = nf_y[t]; h[3 * (size_t)t + 2] = nf_z[t];
  }
  const size_t nd = h.size();
  if (cudaMalloc(&b.surf, sizeof(double) * nd + sizeof(int) * tri.size()) != cudaSuccess) return CB_E_CUDA;
  b.nf = (double *)b.surf;
  b.u = b.nf + 3 * (size_t)n_elmt;
  b.uold = b.u + 3 * (size_t)n_v;
  b.tri = (int *)(b.nf + nd);
  b.n_v = n_v;
  b.n_elmt = n_elmt;
  if (cudaMemcpyAsync(b.nf, h.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b.tri, tri.data(), sizeof(int) * tri.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return CB_E_CUDA;
  return CB_OK;
}

}  // namespace cb
