// Hartree-Fock functional and linear-mixing kernels (device-resident SCF).
#pragma once
#include <cuda_runtime.h>
#include "lqm_team.cuh"

namespace lqm {

// V0 = sum_L v[L] in key order (Meanfield/hartreefock.jl:159).
__global__ void v0_kernel(int64_t nn, int nv, const double2* __restrict__ v, double2* __restrict__ V0) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    double2 s = cmk(0.0, 0.0);
    for (int l = 0; l < nv; ++l) s = cadd(s, v[(int64_t)l * nn + e]);
    V0[e] = s;
  }
}

// hMF[m] = h[hidx[m]] (or 0) - v[fv[m]] .* rho[fr[m]]  (hartreefock.jl:191-205,247-276)
__global__ void hf_build_kernel(int64_t nn, int nm, const int* __restrict__ hidx, const int* __restrict__ fv,
                                const int* __restrict__ fr, const double2* __restrict__ h,
                                const double2* __restrict__ v, const double2* __restrict__ rho,
                                double2* __restrict__ hmf) {
  const int64_t tot = nn * nm;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(t / nn);
    const int64_t e = t % nn;
    double2 val = hidx[m] >= 0 ? h[(int64_t)hidx[m] * nn + e] : cmk(0.0, 0.0);
    if (fv[m] >= 0 && fr[m] >= 0) val = csub(val, cmul(v[(int64_t)fv[m] * nn + e], rho[(int64_t)fr[m] * nn + e]));
    hmf[t] = val;
  }
}

// Hartree shift hMF0[i,i] += (V0 diag(rho0))_i and eH = 1/2 Re(n^T V0 n) (hartreefock.jl:278-289,392-397).
__global__ void hartree_kernel(int n, const double2* __restrict__ V0, const double2* __restrict__ rho0,
                               double2* __restrict__ hmf0, double* __restrict__ eH) {
  __shared__ double red[32];
  const Team T = make_team();
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 d = cmk(0.0, 0.0);
    for (int j = 0; j < n; ++j) d = cadd(d, cmul(V0[i + (int64_t)j * n], rho0[j + (int64_t)j * n]));
    hmf0[i + (int64_t)i * n] = cadd(hmf0[i + (int64_t)i * n], d);
    s += cmul(rho0[i + (int64_t)i * n], d).x;
  }
  s = team_sum(T, s, red);
  if (threadIdx.x == 0) eH[0] = 0.5 * s;
}

// Partial sums of Re(rho .* conj(rho) .* v) over the Fock pairs (hartreefock.jl:405-410).
__global__ void __launch_bounds__(256) fock_energy_partial(int64_t nn, int nf, const int* __restrict__ fv,
                                                           const int* __restrict__ fr, const double2* __restrict__ v,
                                                           const double2* __restrict__ rho, int64_t chunk,
                                                           double* __restrict__ partial) {
  __shared__ double red[32];
  const Team T = make_team();
  const int64_t tot = nn * nf;
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = (b0 + chunk < tot) ? b0 + chunk : tot;
  double s = 0.0;
  for (int64_t t = b0 + threadIdx.x; t < b1; t += blockDim.x) {
    const int f = (int)(t / nn);
    const int64_t e = t % nn;
    const double2 r = rho[(int64_t)fr[f] * nn + e];
    const double2 vv = v[(int64_t)fv[f] * nn + e];
    s += (r.x * r.x + r.y * r.y) * vv.x;
  }
  s = team_sum(T, s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// x1 = beta x1 + (1-beta) x0; partials of |x1-x0|^2 and |x1|^2; x0 = x1 (fixedpoint.jl:146-160).
__global__ void __launch_bounds__(256) mix_kernel(int64_t m, double beta, double2* __restrict__ x1,
                                                  double2* __restrict__ x0, int64_t chunk,
                                                  double* __restrict__ pdiff, double* __restrict__ pnorm) {
  __shared__ double red[32];
  const Team T = make_team();
  const int64_t b0 = blockIdx.x * chunk;
  const int64_t b1 = (b0 + chunk < m) ? b0 + chunk : m;
  double sd = 0.0, sn = 0.0;
  for (int64_t t = b0 + threadIdx.x; t < b1; t += blockDim.x) {
    const double2 a = x1[t], b = x0[t];
    const double2 y = cmk(beta * a.x + (1.0 - beta) * b.x, beta * a.y + (1.0 - beta) * b.y);
    const double dx = y.x - b.x, dy = y.y - b.y;
    sd += dx * dx + dy * dy;
    sn += y.x * y.x + y.y * y.y;
    x1[t] = y;
    x0[t] = y;
  }
  sd = team_sum(T, sd, red);
  sn = team_sum(T, sn, red);
  if (threadIdx.x == 0) { pdiff[blockIdx.x] = sd; pnorm[blockIdx.x] = sn; }
}

// ---- J-augmented Hartree-Fock (ExchangeKernel, hartreefock.jl:24-76,298-381).
// sf[a + ns f] is the orbital of (site a, flavor f); Jtot = sum_L j[L] (ns x ns);
// jb the j blocks (ns x ns each); jr/jm the rho / hMF block of each j key (jr < 0: rho
// lacks the key, the bond field and energy skip it).

// Sigma_loc: H0[(a al), (a be)] -= sum_b Jtot[a, b] rho0[(b al), (b be)], b in order
// (hartreefock.jl:306-314).  One thread per (a, al, be).
__global__ void exch_local_kernel(int n, int ns, int nf, const int* __restrict__ sf, const double2* __restrict__ Jtot,
                                  const double2* __restrict__ rho0, double2* __restrict__ H0) {
  const int64_t tot = (int64_t)ns * nf * nf;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(t / (nf * nf));
    const int r = (int)(t - (int64_t)a * nf * nf);
    const int al = r / nf, be = r - (r / nf) * nf;
    const int64_t o = sf[a + ns * al] + (int64_t)n * sf[a + ns * be];
    double2 acc = H0[o];
    for (int b = 0; b < ns; ++b) {
      const double2 J = Jtot[a + (int64_t)ns * b];
      if (J.x == 0.0 && J.y == 0.0) continue;
      acc = csub(acc, cmul(J, rho0[sf[b + ns * al] + (int64_t)n * sf[b + ns * be]]));
    }
    H0[o] = acc;
  }
}

// Sigma_bond[L][(a al), (b al)] += J_ab(L) tau_L[a, b], tau = sum_al rho_L[(a al), (b al)]
// (hartreefock.jl:316-336).  One thread per (j key, a, b); the written entries are
// distinct across threads.
__global__ void exch_bond_kernel(int n, int ns, int nf, const int* __restrict__ sf, int nJ,
                                 const double2* __restrict__ jb, const int* __restrict__ jr,
                                 const int* __restrict__ jm, const double2* __restrict__ rho,
                                 double2* __restrict__ hmf) {
  const int64_t nn = (int64_t)n * n, ss = (int64_t)ns * ns;
  const int64_t tot = (int64_t)nJ * ss;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(t / ss);
    const int64_t e = t - (int64_t)l * ss;
    if (jr[l] < 0) continue;
    const double2 J = jb[t];
    if (J.x == 0.0 && J.y == 0.0) continue;
    const int a = (int)(e % ns), b = (int)(e / ns);
    const double2* rL = rho + (int64_t)jr[l] * nn;
    double2* hL = hmf + (int64_t)jm[l] * nn;
    double2 tau = cmk(0.0, 0.0);
    for (int al = 0; al < nf; ++al) tau = cadd(tau, rL[sf[a + ns * al] + (int64_t)n * sf[b + ns * al]]);
    const double2 f = cmul(J, tau);
    for (int al = 0; al < nf; ++al) {
      const int64_t o = sf[a + ns * al] + (int64_t)n * sf[b + ns * al];
      hL[o] = cadd(hL[o], f);
    }
  }
}

// eJ = 1/2 Re sum_L sum_ab J_ab(L) (|tau_L[a,b]|^2 - Tr_f[m_a m_b])  (hartreefock.jl:345-381):
// the local part with Jtot over the (a, b) pairs, the bond part over (j key, a, b);
// one CTA, per-thread strided sums and a fixed-order team reduction.
__global__ void exch_energy_kernel(int n, int ns, int nf, const int* __restrict__ sf,
                                   const double2* __restrict__ Jtot, int nJ, const double2* __restrict__ jb,
                                   const int* __restrict__ jr, const double2* __restrict__ rho, int zr,
                                   double* __restrict__ eJ) {
  __shared__ double red[32];
  const Team T = make_team();
  const int64_t nn = (int64_t)n * n, ss = (int64_t)ns * ns;
  const double2* r0 = rho + (int64_t)zr * nn;
  double s = 0.0;
  for (int64_t t = threadIdx.x; t < ss; t += blockDim.x) {
    const int a = (int)(t % ns), b = (int)(t / ns);
    const double2 J = Jtot[t];
    if (J.x == 0.0 && J.y == 0.0) continue;
    double2 tr = cmk(0.0, 0.0);
    for (int al = 0; al < nf; ++al)
      for (int be = 0; be < nf; ++be)
        tr = cadd(tr, cmul(r0[sf[a + ns * al] + (int64_t)n * sf[a + ns * be]],
                           r0[sf[b + ns * be] + (int64_t)n * sf[b + ns * al]]));
    s -= 0.5 * cmul(J, tr).x;
  }
  for (int64_t t = threadIdx.x; t < (int64_t)nJ * ss; t += blockDim.x) {
    const int l = (int)(t / ss);
    if (jr[l] < 0) continue;
    const double2 J = jb[t];
    if (J.x == 0.0 && J.y == 0.0) continue;
    const int64_t e = t - (int64_t)l * ss;
    const int a = (int)(e % ns), b = (int)(e / ns);
    const double2* rL = rho + (int64_t)jr[l] * nn;
    double2 tau = cmk(0.0, 0.0);
    for (int al = 0; al < nf; ++al) tau = cadd(tau, rL[sf[a + ns * al] + (int64_t)n * sf[b + ns * al]]);
    s += 0.5 * J.x * (tau.x * tau.x + tau.y * tau.y);
  }
  s = team_sum(T, s, red);
  if (threadIdx.x == 0) eJ[0] = s;
}

}  // namespace lqm
