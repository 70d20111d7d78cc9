// dda_cuda.hpp -- C++ host classes over the C ABI of dda_cuda.h, shaped like
// the reference's interfaces so reference-style driver code can call the B200
// path unchanged:
//
//   dda::CudaMatVec<T>      MatVec<T> (DDA/MatVec.hpp:33-55): setCoupleConstants,
//                           apply(arg, result, conj) on host vectors of
//                           3*vecStride complex numbers
//   dda::CudaSolver<T>      IterativeSolverBase<T>::getPolVec
//                           (DDA/IterativeSolverBase.hpp:59), solver chosen by
//                           its --iter name (DDA/DDAMain.cpp:647-656)
//
// Errors become dda::Error exceptions, as Core::Exception is thrown by the
// reference (Core/Assert.hpp).  Header only; link with -ldda_b200.
#ifndef DDA_CUDA_HPP
#define DDA_CUDA_HPP

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "dda_cuda.h"
#include "dda_frontend.h"

namespace dda {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const dda_ctx* ctx) {
  if (rc != DDA_OK) throw Error(rc, dda_last_error(ctx));
}

// Precision of the device path for the reference's ftype.
template <typename T> struct Precision;
template <> struct Precision<double> { static const int value = DDA_PREC_FP64; };
template <> struct Precision<float> { static const int value = DDA_PREC_FP32; };

// The device context and matvec.  The problem description (dipole list, box,
// grid, kd) comes from DDAParams; D is generated on the GPU unless given.
template <typename T>
class CudaMatVec {
 public:
  typedef std::complex<T> ctype;

  CudaMatVec(const dda_problem& prob, int precision = Precision<T>::value) {
    check(dda_create(&prob, precision, &ctx_), nullptr);
    nvs_ = (size_t)dda_vec_stride(ctx_);
  }
  ~CudaMatVec() { dda_destroy(ctx_); }
  CudaMatVec(const CudaMatVec&) = delete;
  CudaMatVec& operator=(const CudaMatVec&) = delete;

  size_t vecStride() const { return nvs_; }
  dda_ctx* context() const { return ctx_; }

  // MatVec<T>::setCoupleConstants (DDA/MatVec.hpp:46): cc_sqrt holds
  // nmat*3 values (DiagMatrix3 per material).
  void setCoupleConstants(const std::vector<std::complex<double>>& cc_sqrt, int rhs = 0) {
    check(dda_set_cc(ctx_, rhs, reinterpret_cast<const double*>(cc_sqrt.data())), ctx_);
  }

  // MatVec<T>::apply (DDA/MatVec.hpp:54): result = A arg, or conj(A conj(arg)).
  void apply(const std::vector<ctype>& arg, std::vector<ctype>& result, bool conj) {
    if (arg.size() % (3 * nvs_) != 0) throw Error(DDA_ERR_ARG, "vector size is not a multiple of 3*vecStride");
    const int nrhs = (int)(arg.size() / (3 * nvs_));
    std::vector<std::complex<double>> a(arg.begin(), arg.end()), r(arg.size());
    check(dda_matvec_host(ctx_, reinterpret_cast<const double*>(a.data()), reinterpret_cast<double*>(r.data()),
                          conj ? 1 : 0, nrhs),
          ctx_);
    result.assign(r.begin(), r.end());
  }

 private:
  dda_ctx* ctx_ = nullptr;
  size_t nvs_ = 0;
};

namespace detail {
// dda_solve on the vectors' own precision: complex double, or complex float
// (the --ftype float vectors, dda_solve_f32: no widening copies).
inline int solve(dda_ctx* c, int solver, int nrhs, const std::complex<double>* e, double eps, int64_t maxIter,
                 const std::complex<double>* s, std::complex<double>* p, double* h, int64_t cap, dda_stats* st) {
  return dda_solve(c, solver, nrhs, reinterpret_cast<const double*>(e), eps, maxIter,
                   reinterpret_cast<const double*>(s), reinterpret_cast<double*>(p), h, cap, st);
}
inline int solve(dda_ctx* c, int solver, int nrhs, const std::complex<float>* e, double eps, int64_t maxIter,
                 const std::complex<float>* s, std::complex<float>* p, double* h, int64_t cap, dda_stats* st) {
  return dda_solve_f32(c, solver, nrhs, reinterpret_cast<const float*>(e), eps, maxIter,
                       reinterpret_cast<const float*>(s), reinterpret_cast<float*>(p), h, cap, st);
}
}  // namespace detail

template <typename T>
class CudaSolver {
 public:
  typedef std::complex<T> ctype;

  // name: "qmr", "bicgstab", "bicg" or "cgnr"; maxIter <= 0: unlimited.
  CudaSolver(CudaMatVec<T>& mv, const std::string& name, int64_t maxIter = 0) : mv_(mv), maxIter_(maxIter) {
    if (name == "qmr") solver_ = DDA_SOLVER_QMR;
    else if (name == "bicgstab") solver_ = DDA_SOLVER_BICGSTAB;
    else if (name == "bicg") solver_ = DDA_SOLVER_BICG;
    else if (name == "cgnr") solver_ = DDA_SOLVER_CGNR;
    else throw Error(DDA_ERR_ARG, "Unknown solver `" + name + "'");
  }

  void setCoupleConstants(const std::vector<std::complex<double>>& cc_sqrt, int rhs = 0) {
    mv_.setCoupleConstants(cc_sqrt, rhs);
  }

  // IterativeSolverBase<T>::getPolVec: polarisations for incident field(s)
  // einc (one or more right-hand sides of 3*vecStride values each) solved
  // to relative residual eps; `start` as --load-start-dip-pol.  The relative
  // residual of every iteration is appended to `residuals` (the RE_ lines).
  std::vector<ctype> getPolVec(const std::vector<ctype>& einc, T eps, std::vector<double>* residuals = nullptr,
                               const std::vector<ctype>& start = std::vector<ctype>()) {
    const size_t n = einc.size();
    const int nrhs = (int)(n / (3 * mv_.vecStride()));
    std::vector<ctype> p(n);
    const int64_t cap = 100000;
    std::vector<double> hist(residuals ? (size_t)cap * nrhs : 0);
    stats_.assign(nrhs, dda_stats());
    const int rc = detail::solve(mv_.context(), solver_, nrhs, einc.data(), (double)eps, maxIter_,
                                 start.empty() ? nullptr : start.data(), p.data(), residuals ? hist.data() : nullptr,
                                 residuals ? cap : 0, stats_.data());
    if (residuals)
      for (int r = 0; r < nrhs; r++)
        residuals->insert(residuals->end(), hist.begin() + (size_t)r * cap,
                          hist.begin() + (size_t)r * cap + std::min<int64_t>(cap, stats_[r].iterations));
    check(rc, mv_.context());
    return p;
  }

  const std::vector<dda_stats>& stats() const { return stats_; }

 private:
  CudaMatVec<T>& mv_;
  int solver_ = DDA_SOLVER_QMR;
  int64_t maxIter_;
  std::vector<dda_stats> stats_;
};

}  // namespace dda

#endif  // DDA_CUDA_HPP
