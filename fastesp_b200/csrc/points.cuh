// Evaluation-point generation on the GPU (the steps before the evaluation):
//
//  * vdW surface: n_a Fibonacci points on the sphere of atom a (centre R_a,
//    radius r_a), phi_i = acos(1 - 2(i+1/2)/n_a), theta_i = pi (1+sqrt 5)(i+1/2);
//    a candidate is kept when it lies on the exposed surface, i.e. its distance
//    to every nucleus b is >= r_b - 1e-9 (benchmarks/make_points.py:22-58,
//    examples/vdw_surface_esp.py:38-52).  O(N_candidates x N_atoms).
//  * cubic grid: grid points given by their flat index into an nx x ny x nz grid
//    whose axis coordinates are given (as the host computes them), kept when
//    farther than ``exclude`` from every nucleus.
// Products and sums are rounded one by one (no contraction), as NumPy does.
//
// One thread per candidate writes its point and a keep flag; the kept points
// are then compacted in candidate order with the deterministic scan of the
// table builder, so the output order is that of the host generators.
#pragma once
#include "common.cuh"

struct FePointArgs {
  const double* xyz;        // (natom, 3) nuclei
  const double* rad;        // (natom) sphere radius of each atom (surface mode)
  int natom;
  double slack;             // surface: kept when |C - R_b| >= rad_b - slack for all b
  double excl;              // grid: kept when |C - R_b| >= excl for all b
  // surface mode
  const long long* off;     // (natom + 1) first candidate of each atom
  // grid mode
  const long long* index;   // flat grid indices of the candidates
  const double* axes;       // x[nx], y[ny], z[nz] grid coordinates
  long long nx, ny, nz;
  int grid;                 // 0: surface, 1: grid
  long long ncand;
  double* cand;             // (ncand, 3)
  int* keep;                // (ncand)
};

__global__ void fe_point_candidates_kernel(const FePointArgs a) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= a.ncand) return;
  double c[3];
  if (a.grid) {
    const long long f = a.index[g];
    const long long ix = f / (a.ny * a.nz), rem = f % (a.ny * a.nz);
    const long long iy = rem / a.nz, iz = rem % a.nz;
    c[0] = a.axes[ix];
    c[1] = a.axes[a.nx + iy];
    c[2] = a.axes[a.nx + a.ny + iz];
  } else {
    int lo = 0, hi = a.natom - 1;                 // atom: last with off <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (a.off[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const long long n = a.off[lo + 1] - a.off[lo];
    const double i = double(g - a.off[lo]) + 0.5;
    const double phi = acos(__dsub_rn(1.0, __ddiv_rn(__dmul_rn(2.0, i), double(n))));
    const double theta = __dmul_rn(__dmul_rn(3.14159265358979323846, 1.0 + sqrt(5.0)), i);
    double sp, cp, st, ct;
    sincos(phi, &sp, &cp);
    sincos(theta, &st, &ct);
    const double r = a.rad[lo];
    c[0] = __dadd_rn(a.xyz[3 * lo], __dmul_rn(r, __dmul_rn(sp, ct)));
    c[1] = __dadd_rn(a.xyz[3 * lo + 1], __dmul_rn(r, __dmul_rn(sp, st)));
    c[2] = __dadd_rn(a.xyz[3 * lo + 2], __dmul_rn(r, cp));
  }
  int ok = 1;
  for (int b = 0; b < a.natom && ok; ++b) {
    const double dx = c[0] - a.xyz[3 * b], dy = c[1] - a.xyz[3 * b + 1], dz = c[2] - a.xyz[3 * b + 2];
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    ok = __dsqrt_rn(d2) >= (a.grid ? a.excl : a.rad[b] - a.slack);
  }
  a.cand[3 * g] = c[0];
  a.cand[3 * g + 1] = c[1];
  a.cand[3 * g + 2] = c[2];
  a.keep[g] = ok;
}

// out[pos[g]] = cand[g] for kept candidates; *count = number kept.
__global__ void fe_point_compact_kernel(const double* __restrict__ cand,
                                        const int* __restrict__ keep,
                                        const int* __restrict__ pos, long long ncand,
                                        double* __restrict__ out, long long cap, int* count) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= ncand) return;
  if (g == ncand - 1) *count = pos[g] + keep[g];
  if (!keep[g]) return;
  const long long d = pos[g];
  if (d >= cap) { fe_flag(FE_ST_OVERFLOW); return; }
  out[3 * d] = cand[3 * g];
  out[3 * d + 1] = cand[3 * g + 1];
  out[3 * d + 2] = cand[3 * g + 2];
}
