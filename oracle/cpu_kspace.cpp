// CPU restatement of LatticeQM.jl's `:multithreaded` k-loop for the density
// matrix and the bands (TEST INFRASTRUCTURE ONLY: the checker and the timed CPU
// baseline of bench.py; the product library never links or calls it).
//
// Per k-point, as the reference does it:
//   H(k) = sum_R H_R exp(+i 2 pi k.R) in key order    TightBinding/types.jl:8,18-25
//   eigen!(Hermitian(H(k))) -> LAPACK zheevr,          Eigen/Eigen.jl:22-23,32
//     jobz 'V' (or 'N' for bands), range 'A', uplo 'U', abstol -1
//   f = fermidirac(eps; mu, T) (T = 0: Heaviside, 1/2 at equality)   Utils/fermidirac.jl:1-5
//   rho_k = (U diag f) U^H, two products                Operators/densitymatrix.jl:139-140
//   rho_L += w_k exp(-i 2 pi k.L) rho_k for every key  densitymatrix.jl:141-143
//   eband += w_k sum_j eps_j f_j                        densitymatrix.jl:144
// The k-points are split into contiguous chunks handed out dynamically to the
// threads (Parallel.jl:243-258, ThreadedExec); each thread folds into its own
// partial rho, and the partials are summed in thread order at the end
// (Parallel.jl:289-327).  BLAS runs on one thread per caller thread, as
// Parallel.configure_blas! pins it (Parallel.jl:146-191).
//
// LAPACK/BLAS: the zheevr/zgemm that SciPy ships (its bundled OpenBLAS, symbols
// scipy_zheevr_/scipy_zgemm_), the same routines Julia's LinearAlgebra calls.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

using cd = std::complex<double>;

extern "C" {
void scipy_zheevr_(const char* jobz, const char* range, const char* uplo, const int* n, cd* a, const int* lda,
                   const double* vl, const double* vu, const int* il, const int* iu, const double* abstol, int* m,
                   double* w, cd* z, const int* ldz, int* isuppz, cd* work, const int* lwork, double* rwork,
                   const int* lrwork, int* iwork, const int* liwork, int* info, size_t, size_t, size_t);
void scipy_zgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k, const cd* alpha,
                  const cd* a, const int* lda, const cd* b, const int* ldb, const cd* beta, cd* c, const int* ldc,
                  size_t, size_t);
void scipy_openblas_set_num_threads(int);
}

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

struct Eig {
  int n;
  std::vector<cd> A, Z, work;
  std::vector<double> w, rwork;
  std::vector<int> isuppz, iwork;
  explicit Eig(int n_) : n(n_), A((size_t)n_ * n_), Z((size_t)n_ * n_), w(n_), isuppz(2 * (size_t)n_) {
    // workspace query
    int lwork = -1, lrwork = -1, liwork = -1, m = 0, info = 0, il = 0, iu = 0;
    double vl = 0, vu = 0, abstol = -1.0;
    cd wq;
    double rq;
    int iq;
    scipy_zheevr_("V", "A", "U", &n, A.data(), &n, &vl, &vu, &il, &iu, &abstol, &m, w.data(), Z.data(), &n,
                  isuppz.data(), &wq, &lwork, &rq, &lrwork, &iq, &liwork, &info, 1, 1, 1);
    work.resize((size_t)std::max(1.0, wq.real()));
    rwork.resize((size_t)std::max(1.0, rq));
    iwork.resize((size_t)std::max(1, iq));
  }
  // eigen-decomposition of A (overwritten); vectors into Z when `vec`
  int run(bool vec) {
    int lwork = (int)work.size(), lrwork = (int)rwork.size(), liwork = (int)iwork.size();
    int m = 0, info = 0, il = 0, iu = 0;
    double vl = 0, vu = 0, abstol = -1.0;
    scipy_zheevr_(vec ? "V" : "N", "A", "U", &n, A.data(), &n, &vl, &vu, &il, &iu, &abstol, &m, w.data(),
                  Z.data(), &n, isuppz.data(), work.data(), &lwork, rwork.data(), &lrwork, iwork.data(), &liwork,
                  &info, 1, 1, 1);
    return info;
  }
};

// H(k) = sum_R H_R e^{+i 2 pi k.R}, blocks n x n x nR column-major, keys d x nR.
void fouriersum(int n, int nR, int d, const int64_t* keys, const cd* blocks, const double* k, cd* out) {
  const size_t nn = (size_t)n * n;
  for (int r = 0; r < nR; ++r) {
    double dot = 0.0;
    for (int a = 0; a < d; ++a) dot += k[a] * (double)keys[(size_t)r * d + a];
    const cd ph = std::polar(1.0, kTwoPi * dot);
    const cd* B = blocks + (size_t)r * nn;
    if (r == 0)
      for (size_t i = 0; i < nn; ++i) out[i] = B[i] * ph;
    else
      for (size_t i = 0; i < nn; ++i) out[i] += B[i] * ph;
  }
}

inline double fermidirac(double e, double mu, double T) {
  if (T == 0.0) return e < mu ? 1.0 : (e > mu ? 0.0 : 0.5);
  return 1.0 / (std::exp((e - mu) / T) + 1.0);
}

}  // namespace

extern "C" {

// rho (n x n x nL, overwritten), eband; bands (n x nk) optional.  w NULL = 1/nk.
// Returns 0, or the first nonzero LAPACK info.
int lqm_cpu_densitymatrix(int64_t n64, int64_t nR, int32_t d, const int64_t* keys, const double* blocks_, int64_t nk,
                          const double* ks, const double* w, double mu, double T, int64_t nL, const int64_t* Lkeys,
                          double* rho_, double* eband, double* bands, int nthreads) {
  const int n = (int)n64;
  const size_t nn = (size_t)n * n;
  const cd* blocks = reinterpret_cast<const cd*>(blocks_);
  cd* rho = reinterpret_cast<cd*>(rho_);
  if (nthreads < 1) nthreads = omp_get_max_threads();
  scipy_openblas_set_num_threads(1);
  std::vector<std::vector<cd>> part((size_t)nthreads);
  std::vector<double> ebp((size_t)nthreads, 0.0);
  int err = 0;
  const int64_t chunk = std::max<int64_t>(1, nk / (4 * (int64_t)nthreads));
#pragma omp parallel num_threads(nthreads)
  {
    const int t = omp_get_thread_num();
    std::vector<cd>& P = part[(size_t)t];
    P.assign(nn * (size_t)nL, cd(0.0, 0.0));
    Eig E(n);
    std::vector<cd> X(nn), Rk(nn);
    std::vector<double> f((size_t)n);
    const cd one(1.0, 0.0), zero(0.0, 0.0);
#pragma omp for schedule(dynamic, chunk)
    for (int64_t j = 0; j < nk; ++j) {
      const double* k = ks + (size_t)j * d;
      const double wk = w ? w[j] : 1.0 / (double)nk;
      fouriersum(n, (int)nR, d, keys, blocks, k, E.A.data());
      const int info = E.run(true);
      if (info != 0) {
#pragma omp atomic write
        err = info;
      }
      if (bands) std::memcpy(bands + (size_t)j * n, E.w.data(), (size_t)n * sizeof(double));
      double eb = 0.0;
      for (int i = 0; i < n; ++i) {
        f[(size_t)i] = fermidirac(E.w[(size_t)i], mu, T);
        eb += E.w[(size_t)i] * f[(size_t)i];
      }
      ebp[(size_t)t] += wk * eb;
      for (int c = 0; c < n; ++c)  // tmp = U diag(f)
        for (int i = 0; i < n; ++i) X[(size_t)c * n + i] = E.Z[(size_t)c * n + i] * f[(size_t)c];
      scipy_zgemm_("N", "C", &n, &n, &n, &one, X.data(), &n, E.Z.data(), &n, &zero, Rk.data(), &n, 1, 1);
      for (int64_t l = 0; l < nL; ++l) {
        double dot = 0.0;
        for (int a = 0; a < d; ++a) dot += k[a] * (double)Lkeys[(size_t)l * d + a];
        const cd c = wk * std::polar(1.0, -kTwoPi * dot);
        cd* Pl = P.data() + (size_t)l * nn;
        for (size_t i = 0; i < nn; ++i) Pl[i] += c * Rk[i];
      }
    }
  }
  std::fill(rho, rho + nn * (size_t)nL, cd(0.0, 0.0));
  double eb = 0.0;
  for (int t = 0; t < nthreads; ++t) {
    const std::vector<cd>& P = part[(size_t)t];
    for (size_t i = 0; i < P.size(); ++i) rho[i] += P[i];
    eb += ebp[(size_t)t];
  }
  if (eband) *eband = eb;
  return err;
}

// Bands only (zheevr jobz 'N'), n x nk.
int lqm_cpu_bandmatrix(int64_t n64, int64_t nR, int32_t d, const int64_t* keys, const double* blocks_, int64_t nk,
                       const double* ks, double* bands, int nthreads) {
  const int n = (int)n64;
  const cd* blocks = reinterpret_cast<const cd*>(blocks_);
  if (nthreads < 1) nthreads = omp_get_max_threads();
  scipy_openblas_set_num_threads(1);
  int err = 0;
#pragma omp parallel num_threads(nthreads)
  {
    Eig E(n);
#pragma omp for schedule(dynamic, 1)
    for (int64_t j = 0; j < nk; ++j) {
      fouriersum(n, (int)nR, d, keys, blocks, ks + (size_t)j * d, E.A.data());
      const int info = E.run(false);
      if (info != 0) {
#pragma omp atomic write
        err = info;
      }
      std::memcpy(bands + (size_t)j * n, E.w.data(), (size_t)n * sizeof(double));
    }
  }
  return err;
}

int lqm_cpu_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
