// Reflux at the interfaces of an AMR hierarchy on one rank (GRACE's
// src/evolution/refluxing.cpp:528-1170, the local branches of
// reflux_correct_fluxes and reflux_correct_emfs), driven by the face and
// edge descriptors the caller's forest provides (amr_ghosts.hh:190-330).
//
//  fluxes (after FOFC, before the flux divergence):
//    k_reflux_faces        the coarse block's flux on a hanging face replaced
//                          by the area average of the 4 fine fluxes
//                          (refluxing.cpp:586-621)
//    k_reflux_same_faces   optional: the two same-level blocks' fluxes on a
//                          shared face replaced by their mean (compiled in
//                          the reference with GRACE_SAME_LEVEL_FACE_AVERAGE,
//                          refluxing.cpp:623-686)
//  edge EMFs (after the update, before the CT update):
//    k_reflux_emf_faces    the coarse block's EMFs on the inner lines of a
//                          hanging face replaced by the mean of the two fine
//                          EMFs they cover (refluxing.cpp:720-808)
//    k_reflux_emf_same_faces  both blocks' tangential EMFs on the inner lines
//                          of a same-level face replaced by their mean
//                          (refluxing.cpp:812-937)
//    k_reflux_emf_edges_*  hanging edges (where blocks of two levels meet
//                          along an edge, and the middle lines of hanging
//                          faces): the fine EMFs of the fine side with the
//                          smallest edge id become every side's value, the
//                          coarse sides taking the mean of the two fine cells
//                          their cell covers (refluxing.cpp:944-1056)
//    k_reflux_emf_same_edges_*  same-level edges: every side takes the value
//                          of the side with the smallest edge id
//                          (refluxing.cpp:1065-1140)
// Blocks are cubic (n cells a side).  Every sum is written in the
// reference's order and each value rounded on its own, so the results are
// the reference's bit for bit.
#pragma once
#include "stage_kernels.cuh"

namespace grb {

// other_dirs of refluxing.cpp: the two axes orthogonal to an axis, in order
__device__ __forceinline__ int odir(int axis, int which) {
  return which == 0 ? (axis == 0 ? 1 : 0) : (axis == 2 ? 1 : 2);
}

// Device view of the caller's descriptor lists (grb_reflux).
struct RefluxDev {
  int64_t nfaces;
  const int64_t* face_cq;   // [nfaces]
  const uint8_t* face_cid;  // [nfaces]
  const int64_t* face_fq;   // [nfaces][4]
  int64_t nsame;
  const int64_t* same_q;    // [nsame][2]
  const uint8_t* same_id;   // [nsame][2]
  int64_t nedges;
  const uint8_t* edge_ns;   // [nedges]
  const uint8_t* edge_id;   // [nedges][4]
  const uint8_t* edge_fine; // [nedges][4]
  const int64_t* edge_q;    // [nedges][4][2]
  const uint8_t* edge_off;  // [nedges][4][2]
  int64_t nsame_edges;
  const uint8_t* sedge_ns;  // [n]
  const uint8_t* sedge_id;  // [n][4]
  const int64_t* sedge_q;   // [n][4]
  double* acc_edges;        // [nedges][2][n] accumulation (handle scratch)
  double* acc_same_edges;   // [nsame_edges][n]
};

// (i, j, v, iq) over n x n x 7 x nfaces
__global__ void __launch_bounds__(128) k_reflux_faces(Geo G, RefluxDev R, double* __restrict__ flux) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  const int64_t total = (int64_t)n * n * GRB_N_HRSC * R.nfaces;
  if (t >= total) return;
  const int i = (int)(t % n), j = (int)((t / n) % n);
  const int v = (int)((t / ((int64_t)n * n)) % GRB_N_HRSC);
  const int64_t iq = t / ((int64_t)n * n * GRB_N_HRSC);
  const int64_t qc = R.face_cq[iq];
  const int face = R.face_cid[iq];
  const int dir = face / 2;
  int c[3];
  c[dir] = (face & 1) ? G.g + n : G.g;
  c[odir(dir, 0)] = G.g + i;
  c[odir(dir, 1)] = G.g + j;
  const int child = (2 * i >= n) + 2 * (2 * j >= n);
  const int64_t qf = R.face_fq[4 * iq + child];
  int f[3];
  f[dir] = (face & 1) ? G.g : G.g + n;  // the fine side's face is the opposite one
  f[odir(dir, 0)] = G.g + (2 * i) % n;
  f[odir(dir, 1)] = G.g + (2 * j) % n;
  double s = 0.0;
  for (int ii = 0; ii <= (dir != 0); ++ii)
    for (int jj = 0; jj <= (dir != 1); ++jj)
      for (int kk = 0; kk <= (dir != 2); ++kk) s = __dadd_rn(s, flux[flx(G, f[0] + ii, f[1] + jj, f[2] + kk, v, dir, qf)]);
  flux[flx(G, c[0], c[1], c[2], v, dir, qc)] = __dmul_rn(s, 0.25);
}

// (i, j, v, iq) over n x n x 7 x nsame
__global__ void __launch_bounds__(128) k_reflux_same_faces(Geo G, RefluxDev R, double* __restrict__ flux) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * n * GRB_N_HRSC * R.nsame) return;
  const int i = (int)(t % n), j = (int)((t / n) % n);
  const int v = (int)((t / ((int64_t)n * n)) % GRB_N_HRSC);
  const int64_t iq = t / ((int64_t)n * n * GRB_N_HRSC);
  int64_t at[2];
  double s = 0.0;
  for (int is = 0; is < 2; ++is) {
    const int fid = R.same_id[2 * iq + is], fdir = fid / 2;
    int c[3];
    c[fdir] = (fid & 1) ? n + G.g : G.g;
    c[odir(fdir, 0)] = G.g + i;
    c[odir(fdir, 1)] = G.g + j;
    at[is] = flx(G, c[0], c[1], c[2], v, fdir, R.same_q[2 * iq + is]);
    s = __dadd_rn(s, flux[at[is]]);
  }
  s = __dmul_rn(s, 0.5);
  flux[at[0]] = s;
  flux[at[1]] = s;
}

// (i, j, iq) over (n/2) x (n/2) x nfaces
__global__ void __launch_bounds__(128) k_reflux_emf_faces(Geo G, RefluxDev R, double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx, h = n / 2;
  if (t >= (int64_t)h * h * R.nfaces) return;
  const int i = (int)(t % h), j = (int)((t / h) % h);
  const int64_t iq = t / ((int64_t)h * h);
  const int face = R.face_cid[iq];
  const int fdir = face / 2, idir = odir(fdir, 0), jdir = odir(fdir, 1);
  const int side = face & 1;
  const int64_t qc = R.face_cq[iq];
  for (int ch = 0; ch < 4; ++ch) {
    const int64_t qf = R.face_fq[4 * iq + ch];
    int f[3];
    f[fdir] = side ? G.g : n + G.g;
    f[idir] = 2 * i + G.g;
    f[jdir] = 2 * j + G.g;
    const double ei = __dmul_rn(0.5, __dadd_rn(emf[emi(G, f[0], f[1], f[2], idir, qf)],
                                                emf[emi(G, f[0] + (idir == 0), f[1] + (idir == 1), f[2] + (idir == 2), idir, qf)]));
    const double ej = __dmul_rn(0.5, __dadd_rn(emf[emi(G, f[0], f[1], f[2], jdir, qf)],
                                                emf[emi(G, f[0] + (jdir == 0), f[1] + (jdir == 1), f[2] + (jdir == 2), jdir, qf)]));
    int c[3];
    c[fdir] = side ? n + G.g : G.g;
    c[idir] = i + ((ch & 1) ? h : 0) + G.g;
    c[jdir] = j + ((ch & 2) ? h : 0) + G.g;
    // the face's boundary lines and its two middle lines belong to the
    // edge descriptors
    if (c[jdir] != h + G.g && c[jdir] != G.g) emf[emi(G, c[0], c[1], c[2], idir, qc)] = ei;
    if (c[idir] != h + G.g && c[idir] != G.g) emf[emi(G, c[0], c[1], c[2], jdir, qc)] = ej;
  }
}

// (i, j, iq) over n x n x nsame
__global__ void __launch_bounds__(128) k_reflux_emf_same_faces(Geo G, RefluxDev R, double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * n * R.nsame) return;
  const int i = (int)(t % n), j = (int)((t / n) % n);
  const int64_t iq = t / ((int64_t)n * n);
  double s0 = 0.0, s1 = 0.0;
  int64_t a0[2], a1[2];
  bool w0[2], w1[2];
  for (int is = 0; is < 2; ++is) {
    const int fid = R.same_id[2 * iq + is], fdir = fid / 2, idir = odir(fdir, 0), jdir = odir(fdir, 1);
    const int64_t q = R.same_q[2 * iq + is];
    int c[3];
    c[fdir] = (fid & 1) ? n + G.g : G.g;
    c[idir] = G.g + i;
    c[jdir] = G.g + j;
    a0[is] = emi(G, c[0], c[1], c[2], idir, q);
    a1[is] = emi(G, c[0], c[1], c[2], jdir, q);
    w0[is] = c[jdir] > G.g;
    w1[is] = c[idir] > G.g;
    s0 = __dadd_rn(s0, emf[a0[is]]);
    s1 = __dadd_rn(s1, emf[a1[is]]);
  }
  s0 = __dmul_rn(s0, 0.5);
  s1 = __dmul_rn(s1, 0.5);
  for (int is = 0; is < 2; ++is) {
    if (w0[is]) emf[a0[is]] = s0;
    if (w1[is]) emf[a1[is]] = s1;
  }
}

// Edge cell (i along the edge) of edge `eid` of a block: offsets of the two
// other axes (the block's boundary on each side, or its middle with off).
__device__ __forceinline__ int64_t edge_cell(const Geo& G, int eid, int i, bool off_i, bool off_j, int64_t q) {
  const int n = G.nx, edir = eid / 4;
  int c[3];
  c[edir] = G.g + i;
  c[odir(edir, 0)] = off_i ? n / 2 + G.g : ((eid & 1) ? n + G.g : G.g);
  c[odir(edir, 1)] = off_j ? n / 2 + G.g : (((eid >> 1) & 1) ? n + G.g : G.g);
  return emi(G, c[0], c[1], c[2], edir, q);
}

// (i, iq) over n x nedges: the fine side with the smallest edge id
__global__ void __launch_bounds__(128) k_reflux_emf_edges_compute(Geo G, RefluxDev R, const double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * R.nedges) return;
  const int i = (int)(t % n);
  const int64_t iq = t / n;
  const int ns = R.edge_ns[iq];
  int best = 256;
  double v0 = 0.0, v1 = 0.0;
  for (int s = 0; s < ns; ++s) {
    if (!R.edge_fine[4 * iq + s]) continue;
    const int eid = R.edge_id[4 * iq + s];
    if (eid >= best) continue;
    best = eid;
    v0 = emf[edge_cell(G, eid, i, false, false, R.edge_q[8 * iq + 2 * s])];
    v1 = emf[edge_cell(G, eid, i, false, false, R.edge_q[8 * iq + 2 * s + 1])];
  }
  R.acc_edges[(2 * iq) * n + i] = v0;
  R.acc_edges[(2 * iq + 1) * n + i] = v1;
}
__global__ void __launch_bounds__(128) k_reflux_emf_edges_apply(Geo G, RefluxDev R, double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * R.nedges) return;
  const int i = (int)(t % n);
  const int64_t iq = t / n;
  const int ns = R.edge_ns[iq];
  const double* acc = R.acc_edges + 2 * iq * n;
  for (int s = 0; s < ns; ++s) {
    const int eid = R.edge_id[4 * iq + s];
    if (!R.edge_fine[4 * iq + s]) {
      const int ch = (2 * i) >= n;
      const int a = (2 * i) % n;
      emf[edge_cell(G, eid, i, R.edge_off[8 * iq + 2 * s] != 0, R.edge_off[8 * iq + 2 * s + 1] != 0,
                    R.edge_q[8 * iq + 2 * s])] = __dmul_rn(0.5, __dadd_rn(acc[ch * n + a], acc[ch * n + a + 1]));
    } else {
      for (int ch = 0; ch < 2; ++ch)
        emf[edge_cell(G, eid, i, false, false, R.edge_q[8 * iq + 2 * s + ch])] = acc[ch * n + i];
    }
  }
}

// (i, iq) over n x nsame_edges: the side with the smallest edge id
__global__ void __launch_bounds__(128) k_reflux_emf_same_edges_compute(Geo G, RefluxDev R,
                                                                       const double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * R.nsame_edges) return;
  const int i = (int)(t % n);
  const int64_t iq = t / n;
  const int ns = R.sedge_ns[iq];
  int best = 256;
  double v = 0.0;
  for (int s = 0; s < ns; ++s) {
    const int eid = R.sedge_id[4 * iq + s];
    if (eid >= best) continue;
    best = eid;
    v = emf[edge_cell(G, eid, i, false, false, R.sedge_q[4 * iq + s])];
  }
  R.acc_same_edges[iq * n + i] = v;
}
__global__ void __launch_bounds__(128) k_reflux_emf_same_edges_apply(Geo G, RefluxDev R, double* __restrict__ emf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = G.nx;
  if (t >= (int64_t)n * R.nsame_edges) return;
  const int i = (int)(t % n);
  const int64_t iq = t / n;
  const int ns = R.sedge_ns[iq];
  for (int s = 0; s < ns; ++s)
    emf[edge_cell(G, R.sedge_id[4 * iq + s], i, false, false, R.sedge_q[4 * iq + s])] = R.acc_same_edges[iq * n + i];
}

}  // namespace grb
