// Stand-in for the reference's <DDA/MatVec.hpp> and what it pulls in, for
// compiling the MatVecB200 binding of INTEGRATION.md without the reference
// tree (which needs Boost, FFTW3 and HDF5).  It declares only the members
// that binding uses, with the reference's names and signatures:
//   DDA::DDAParams<T>      nvCount, dipoleGeometry, gridX/Y/Z, kd, gridUnit
//                          (DDA/DDAParams.hpp:115-143)
//   DDA::DipoleGeometry    getGridCoordinates, box, materialIndices,
//                          materials (DDA/DipoleGeometry.hpp:74-149)
//   DDA::CoupleConstants   cc_sqrt (DDA/DDAParams.hpp:223-242)
//   DDA::MatVec<T>         ctor, setCoupleConstants, apply (DDA/MatVec.hpp:33-55)
//   ABORT_MSG, boost::shared_ptr, Core::ProfilingDataPtr
// The bodies are placeholders; nothing here computes.
#ifndef DDA_STUB_MATVEC_HPP
#define DDA_STUB_MATVEC_HPP

#include <complex>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <stdint.h>
#include <vector>

namespace boost { using std::shared_ptr; }
namespace Core {
struct ProfilingData {};
typedef boost::shared_ptr<ProfilingData> ProfilingDataPtr;
}
#define ABORT_MSG(m) throw std::runtime_error(m)

namespace Math {
template <typename T> struct Vector3 {
  T v[3];
  T& operator[](size_t i) { return v[i]; }
  const T& operator[](size_t i) const { return v[i]; }
};
template <typename T> struct DiagMatrix3 {
  T v[3];
  const T& operator[](size_t i) const { return v[i]; }
};
}  // namespace Math

namespace DDA {
// checked integer of the reference (Core/CheckedInteger.hpp): value via ()
struct cuint32_t {
  uint32_t v;
  uint32_t operator()() const { return v; }
};

struct DipoleGeometry {
  std::vector<Math::Vector3<uint32_t> > positions_;
  std::vector<uint8_t> materialIndices_;
  std::vector<Math::DiagMatrix3<std::complex<long double> > > materials_;
  Math::Vector3<cuint32_t> box_;
  Math::Vector3<uint32_t> getGridCoordinates(size_t index) const { return positions_[index]; }
  Math::Vector3<cuint32_t> box() const { return box_; }
  const std::vector<uint8_t>& materialIndices() const { return materialIndices_; }
  const std::vector<Math::DiagMatrix3<std::complex<long double> > >& materials() const { return materials_; }
};

template <typename T> struct DDAParams {
  DipoleGeometry geom_;
  uint32_t nv_, g_[3];
  T kd_, d_;
  const DipoleGeometry& dipoleGeometry() const { return geom_; }
  uint32_t nvCount() const { return nv_; }
  uint32_t gridX() const { return g_[0]; }
  uint32_t gridY() const { return g_[1]; }
  uint32_t gridZ() const { return g_[2]; }
  T kd() const { return kd_; }
  T gridUnit() const { return d_; }
};

template <typename T> struct CoupleConstants {
  std::vector<Math::DiagMatrix3<std::complex<T> > > cc_sqrt_;
  const std::vector<Math::DiagMatrix3<std::complex<T> > >& cc_sqrt() const { return cc_sqrt_; }
};

template <typename T> class MatVec {
  const DDAParams<T>& ddaParams_;
  boost::shared_ptr<const CoupleConstants<T> > cc_;

 public:
  explicit MatVec(const DDAParams<T>& p) : ddaParams_(p) {}
  virtual ~MatVec() {}
  virtual void setCoupleConstants(const boost::shared_ptr<const CoupleConstants<T> >& cc) { cc_ = cc; }
  const DDAParams<T>& g() const { return ddaParams_; }
  virtual void apply(const std::vector<std::complex<T> >& arg, std::vector<std::complex<T> >& result, bool conj,
                     Core::ProfilingDataPtr prof = Core::ProfilingDataPtr()) = 0;
};
}  // namespace DDA

#endif
