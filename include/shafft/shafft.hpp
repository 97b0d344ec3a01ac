// shafft.hpp -- C++ RAII interface of SHAFFT, B200 (sm_100a) backend.
//
// Class and function names, signatures and status semantics follow the
// reference's include/shafft/shafft.hpp:51-1150 (SHAFFT project) so that
// C++ callers and the reference's own tests compile unchanged against this
// header; the GPU-typed overloads take CUDA types (cuFloatComplex,
// cuDoubleComplex, cudaStream_t) where the reference takes HIP types.
#ifndef SHAFFT_CPP_H
#define SHAFFT_CPP_H

#include <shafft/detail/fft_base.hpp>
#include <shafft/shafft.h>
#include <shafft/shafft_config.h>
#include <shafft/shafft_types.hpp>

#include <cstddef>
#include <mpi.h>
#include <vector>

#if SHAFFT_BACKEND_SM100
#include <cuComplex.h>
#include <cuda_runtime_api.h>
#endif

namespace shafft::detail {
class PlanBase;
struct FFT1DPlan;
struct FFTNDPlan;
}  // namespace shafft::detail

namespace shafft {

/// N-dimensional C2C/Z2Z plan.  Flow: configurationND() -> init() ->
/// allocSize()/setBuffers() -> plan() -> execute()/normalize().
class FFTND : public FFT {
public:
  FFTND() noexcept = default;
  ~FFTND() noexcept override;
  void release() noexcept override;
  FFTND(FFTND&& other) noexcept;
  FFTND& operator=(FFTND&& other) noexcept;
  FFTND(const FFTND&) = delete;
  FFTND& operator=(const FFTND&) = delete;

  [[nodiscard]] int init(const std::vector<int>& commDims, const std::vector<size_t>& dimensions,
                         FFTType type, MPI_Comm comm,
                         TransformLayout output = TransformLayout::REDISTRIBUTED) noexcept;
  [[nodiscard]] int plan() noexcept override;
  [[nodiscard]] int setBuffers(complexf* data, complexf* work) noexcept;
  [[nodiscard]] int setBuffers(complexd* data, complexd* work) noexcept;
  [[nodiscard]] int getBuffers(complexf** data, complexf** work) noexcept;
  [[nodiscard]] int getBuffers(complexd** data, complexd** work) noexcept;
#if SHAFFT_BACKEND_SM100
  [[nodiscard]] int setBuffers(cuFloatComplex* data, cuFloatComplex* work) noexcept;
  [[nodiscard]] int setBuffers(cuDoubleComplex* data, cuDoubleComplex* work) noexcept;
  [[nodiscard]] int getBuffers(cuFloatComplex** data, cuFloatComplex** work) noexcept;
  [[nodiscard]] int getBuffers(cuDoubleComplex** data, cuDoubleComplex** work) noexcept;
#endif
  [[nodiscard]] int execute(FFTDirection direction) noexcept override;
  [[nodiscard]] int normalize() noexcept override;
  /// execute(direction) followed by normalize(), fused into the same passes
  /// (extension; no counterpart in the reference).
  [[nodiscard]] int executeNormalized(FFTDirection direction) noexcept;
  [[nodiscard]] size_t allocSize() const noexcept override;
  [[nodiscard]] size_t globalSize() const noexcept override;
  [[nodiscard]] int ndim() const noexcept override;
  [[nodiscard]] FFTType fftType() const noexcept override;
  [[nodiscard]] int getLayout(std::vector<size_t>& subsize, std::vector<size_t>& offset,
                              TensorLayout layout = TensorLayout::CURRENT) const noexcept;
  [[nodiscard]] int getAxes(std::vector<int>& ca, std::vector<int>& da,
                            TensorLayout layout = TensorLayout::CURRENT) const noexcept;
  [[nodiscard]] bool isActive() const noexcept override;
  [[nodiscard]] int setBuffersRaw(void* data, void* work) noexcept override;
  [[nodiscard]] int getBuffersRaw(void** data, void** work) noexcept override;
#if SHAFFT_BACKEND_SM100
  [[nodiscard]] int setStream(cudaStream_t stream) noexcept override;
#endif
  [[nodiscard]] int getCommunicator(MPI_Comm* outComm) const noexcept;
  [[nodiscard]] int init(shafft_nd_config_t& cfg) noexcept;

private:
  detail::FFTNDPlan* data_ = nullptr;
};

/// 1-dimensional C2C/Z2Z plan of global length N (block layout; one rank
/// holds [0, N)).
class FFT1D : public FFT {
public:
  FFT1D() noexcept = default;
  ~FFT1D() noexcept override;
  void release() noexcept override;
  FFT1D(FFT1D&& other) noexcept;
  FFT1D& operator=(FFT1D&& other) noexcept;
  FFT1D(const FFT1D&) = delete;
  FFT1D& operator=(const FFT1D&) = delete;

  [[nodiscard]] int init(size_t globalN, size_t localN, size_t localStart, FFTType precision,
                         MPI_Comm comm) noexcept;
  [[nodiscard]] int plan() noexcept override;
  [[nodiscard]] int setBuffers(complexf* data, complexf* work) noexcept;
  [[nodiscard]] int setBuffers(complexd* data, complexd* work) noexcept;
  [[nodiscard]] int getBuffers(complexf** data, complexf** work) noexcept;
  [[nodiscard]] int getBuffers(complexd** data, complexd** work) noexcept;
#if SHAFFT_BACKEND_SM100
  [[nodiscard]] int setBuffers(cuFloatComplex* data, cuFloatComplex* work) noexcept;
  [[nodiscard]] int setBuffers(cuDoubleComplex* data, cuDoubleComplex* work) noexcept;
  [[nodiscard]] int getBuffers(cuFloatComplex** data, cuFloatComplex** work) noexcept;
  [[nodiscard]] int getBuffers(cuDoubleComplex** data, cuDoubleComplex** work) noexcept;
#endif
  [[nodiscard]] int execute(FFTDirection direction) noexcept override;
  [[nodiscard]] int normalize() noexcept override;
  /// execute(direction) followed by normalize(), fused (extension).
  [[nodiscard]] int executeNormalized(FFTDirection direction) noexcept;
  [[nodiscard]] std::vector<size_t> globalShape() const noexcept;
  [[nodiscard]] size_t globalSize() const noexcept override;
  [[nodiscard]] int ndim() const noexcept override;
  [[nodiscard]] FFTType fftType() const noexcept override;
  [[nodiscard]] size_t localSize() const noexcept;
  [[nodiscard]] size_t allocSize() const noexcept override;
  [[nodiscard]] int getLayout(std::vector<size_t>& localShape, std::vector<size_t>& offset,
                              TensorLayout layout = TensorLayout::CURRENT) const noexcept;
  [[nodiscard]] int getAxes(std::vector<int>& ca, std::vector<int>& da,
                            TensorLayout layout = TensorLayout::CURRENT) const noexcept;
  [[nodiscard]] bool isActive() const noexcept override;
  [[nodiscard]] int setBuffersRaw(void* data, void* work) noexcept override;
  [[nodiscard]] int getBuffersRaw(void** data, void** work) noexcept override;
#if SHAFFT_BACKEND_SM100
  [[nodiscard]] int setStream(cudaStream_t stream) noexcept override;
#endif
  [[nodiscard]] int getCommunicator(MPI_Comm* outComm) const noexcept;
  [[nodiscard]] int init(shafft_1d_config_t& cfg) noexcept;

private:
  detail::FFT1DPlan* data_ = nullptr;
};

#if SHAFFT_BACKEND_SM100
int setStream(detail::PlanBase* plan, cudaStream_t stream);
int getBuffers(detail::PlanBase* plan, cuFloatComplex** data, cuFloatComplex** work) noexcept;
int getBuffers(detail::PlanBase* plan, cuDoubleComplex** data, cuDoubleComplex** work) noexcept;
int setBuffers(detail::PlanBase* plan, cuFloatComplex* data, cuFloatComplex* work) noexcept;
int setBuffers(detail::PlanBase* plan, cuDoubleComplex* data, cuDoubleComplex* work) noexcept;
#endif
int setBuffers(detail::PlanBase* plan, complexf* data, complexf* work) noexcept;
int setBuffers(detail::PlanBase* plan, complexd* data, complexd* work) noexcept;
int getBuffers(detail::PlanBase* plan, complexf** data, complexf** work) noexcept;
int getBuffers(detail::PlanBase* plan, complexd** data, complexd** work) noexcept;

/// Device memory helpers (cudaMalloc / cudaFree / cudaMemcpy).
int allocBuffer(size_t count, complexf** buf) noexcept;
int allocBuffer(size_t count, complexd** buf) noexcept;
int freeBuffer(complexf* buf) noexcept;
int freeBuffer(complexd* buf) noexcept;
int copyToBuffer(complexf* dst, const complexf* src, size_t count) noexcept;
int copyToBuffer(complexd* dst, const complexd* src, size_t count) noexcept;
int copyFromBuffer(complexf* dst, const complexf* src, size_t count) noexcept;
int copyFromBuffer(complexd* dst, const complexd* src, size_t count) noexcept;

int planNDCreate(detail::FFTNDPlan** out);
int FFT1DCreate(detail::FFT1DPlan** out);
int configurationND(const std::vector<size_t>& size, FFTType precision, std::vector<int>& commDims,
                    int& nda, std::vector<size_t>& subsize, std::vector<size_t>& offset,
                    int& commSize, DecompositionStrategy strategy, size_t memLimit, MPI_Comm comm);
int configuration1D(size_t globalN, size_t& localN, size_t& localStart, FFTType precision,
                    MPI_Comm comm);
int planND(detail::FFTNDPlan* plan, const std::vector<int>& commDims,
           const std::vector<size_t>& dimensions, FFTType precision, MPI_Comm comm);
int destroy(detail::PlanBase** plan);
int getLayout(const detail::PlanBase* plan, std::vector<size_t>& subsize,
              std::vector<size_t>& offset, TensorLayout layout);
int getAxes(const detail::PlanBase* plan, std::vector<int>& ca, std::vector<int>& da,
            TensorLayout layout);
int getAllocSize(const detail::PlanBase* plan, size_t& localAllocSize);
int execute(detail::PlanBase* plan, FFTDirection direction);
int normalize(detail::PlanBase* plan);

inline const char* getBackendName() noexcept { return shafftGetBackendName(); }

struct Version {
  int major;
  int minor;
  int patch;
};
inline Version getVersion() noexcept {
  return {SHAFFT_VERSION_MAJOR, SHAFFT_VERSION_MINOR, SHAFFT_VERSION_PATCH};
}
inline const char* getVersionString() noexcept {
  return SHAFFT_STRINGIFY(SHAFFT_VERSION_MAJOR) "." SHAFFT_STRINGIFY(
      SHAFFT_VERSION_MINOR) "." SHAFFT_STRINGIFY(SHAFFT_VERSION_PATCH) SHAFFT_VERSION_SUFFIX;
}

[[nodiscard]] int finalize() noexcept;

/// Owning wrapper of shafft_nd_config_t.
class ConfigND {
public:
  ConfigND(const std::vector<size_t>& globalShape, FFTType precision,
           const std::vector<int>& commDims = {}, int hintNda = 0,
           DecompositionStrategy strategy = DecompositionStrategy::MAXIMIZE_NDA,
           TransformLayout outputPolicy = TransformLayout::REDISTRIBUTED, size_t memLimit = 0,
           MPI_Comm comm = MPI_COMM_WORLD) noexcept;
  ConfigND(const ConfigND&) = delete;
  ConfigND& operator=(const ConfigND&) = delete;
  ConfigND(ConfigND&& other) noexcept;
  ConfigND& operator=(ConfigND&& other) noexcept;
  ~ConfigND() noexcept;
  [[nodiscard]] int status() const noexcept { return status_; }
  [[nodiscard]] const shafft_nd_config_t& cStruct() const noexcept { return cfg_; }
  [[nodiscard]] shafft_nd_config_t& cStruct() noexcept { return cfg_; }
  [[nodiscard]] const shafft_nd_config_t* operator->() const noexcept { return &cfg_; }
  [[nodiscard]] shafft_nd_config_t* operator->() noexcept { return &cfg_; }
  [[nodiscard]] int resolve() noexcept;
  [[nodiscard]] bool isResolved() const noexcept { return (cfg_.flags & SHAFFT_CONFIG_RESOLVED) != 0; }

private:
  shafft_nd_config_t cfg_ = {};
  int status_ = -1;
};

/// Owning wrapper of shafft_1d_config_t.
class Config1D {
public:
  Config1D(size_t globalSize, FFTType precision, MPI_Comm comm) noexcept;
  Config1D(const Config1D&) = delete;
  Config1D& operator=(const Config1D&) = delete;
  Config1D(Config1D&& other) noexcept;
  Config1D& operator=(Config1D&& other) noexcept;
  ~Config1D() noexcept;
  [[nodiscard]] int status() const noexcept { return status_; }
  [[nodiscard]] const shafft_1d_config_t& cStruct() const noexcept { return cfg_; }
  [[nodiscard]] shafft_1d_config_t& cStruct() noexcept { return cfg_; }
  [[nodiscard]] const shafft_1d_config_t* operator->() const noexcept { return &cfg_; }
  [[nodiscard]] shafft_1d_config_t* operator->() noexcept { return &cfg_; }
  [[nodiscard]] int resolve() noexcept;
  [[nodiscard]] bool isResolved() const noexcept { return (cfg_.flags & SHAFFT_CONFIG_RESOLVED) != 0; }

private:
  shafft_1d_config_t cfg_ = {};
  int status_ = -1;
};

}  // namespace shafft

#endif  // SHAFFT_CPP_H
