// Index arithmetic for GRACE's LayoutLeft block arrays and the library's
// face-grid scratch, shared by all kernels.
//
//   cell array (NX,NY,NZ,nv,nq):       i + NX*(j + NY*(k + NZ*(v + nv*q)))
//   face-staggered B (GRACE):          x: (NX+1,NY,NZ), y: (NX,NY+1,NZ), z: (NX,NY,NZ+1)
//   face-grid scratch (FX,FY,FZ,...):  FX = NX+1 etc.; fluxes (.,7,3,nq),
//                                      Eface (.,2,3,nq), vbar (.,4,3,nq),
//                                      emf (.,3,nq), FOFC tags (.,3,nq)
#pragma once
#include <cstdint>

namespace grb {

struct Geo {
  int nx, ny, nz, g;
  int NX, NY, NZ, FX, FY, FZ;
  int64_t nq;
  int64_t cells, fcells;  // per block
};

inline Geo make_geo(int nx, int ny, int nz, int g, int64_t nq) {
  Geo o;
  o.nx = nx; o.ny = ny; o.nz = nz; o.g = g; o.nq = nq;
  o.NX = nx + 2 * g; o.NY = ny + 2 * g; o.NZ = nz + 2 * g;
  o.FX = o.NX + 1; o.FY = o.NY + 1; o.FZ = o.NZ + 1;
  o.cells = (int64_t)o.NX * o.NY * o.NZ;
  o.fcells = (int64_t)o.FX * o.FY * o.FZ;
  return o;
}

__device__ __forceinline__ int64_t cidx(const Geo& G, int i, int j, int k) {
  return (int64_t)i + (int64_t)G.NX * (j + (int64_t)G.NY * k);
}
__device__ __forceinline__ int64_t cvar(const Geo& G, int i, int j, int k, int v, int nv, int64_t q) {
  return cidx(G, i, j, k) + G.cells * ((int64_t)v + (int64_t)nv * q);
}
__device__ __forceinline__ int64_t bxi(const Geo& G, int i, int j, int k, int64_t q) {
  return (int64_t)i + (int64_t)(G.NX + 1) * (j + (int64_t)G.NY * (k + (int64_t)G.NZ * q));
}
__device__ __forceinline__ int64_t byi(const Geo& G, int i, int j, int k, int64_t q) {
  return (int64_t)i + (int64_t)G.NX * (j + (int64_t)(G.NY + 1) * (k + (int64_t)G.NZ * q));
}
__device__ __forceinline__ int64_t bzi(const Geo& G, int i, int j, int k, int64_t q) {
  return (int64_t)i + (int64_t)G.NX * (j + (int64_t)G.NY * (k + (int64_t)(G.NZ + 1) * q));
}
__device__ __forceinline__ int64_t fidx(const Geo& G, int i, int j, int k) {
  return (int64_t)i + (int64_t)G.FX * (j + (int64_t)G.FY * k);
}
// fluxes(i,j,k,v,dir,q)
__device__ __forceinline__ int64_t flx(const Geo& G, int i, int j, int k, int v, int dir, int64_t q) {
  return fidx(G, i, j, k) + G.fcells * ((int64_t)v + 7 * ((int64_t)dir + 3 * q));
}
// Eface(i,j,k,c,dir,q), c in [0,2)
__device__ __forceinline__ int64_t efi(const Geo& G, int i, int j, int k, int c, int dir, int64_t q) {
  return fidx(G, i, j, k) + G.fcells * ((int64_t)c + 2 * ((int64_t)dir + 3 * q));
}
// vbar(i,j,k,c,dir,q), c in [0,4)
__device__ __forceinline__ int64_t vbi(const Geo& G, int i, int j, int k, int c, int dir, int64_t q) {
  return fidx(G, i, j, k) + G.fcells * ((int64_t)c + 4 * ((int64_t)dir + 3 * q));
}
// emf(i,j,k,c,q) and FOFC tags(i,j,k,dir,q)
__device__ __forceinline__ int64_t emi(const Geo& G, int i, int j, int k, int c, int64_t q) {
  return fidx(G, i, j, k) + G.fcells * ((int64_t)c + 3 * q);
}
// Ecenter(i,j,k,c,q)
__device__ __forceinline__ int64_t eci(const Geo& G, int i, int j, int k, int c, int64_t q) {
  return cidx(G, i, j, k) + G.cells * ((int64_t)c + 3 * q);
}

}  // namespace grb
