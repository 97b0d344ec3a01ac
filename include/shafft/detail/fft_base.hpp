// Abstract base of the RAII plan classes (reference include/shafft/detail/fft_base.hpp:23-156).
#ifndef SHAFFT_FFT_BASE_HPP
#define SHAFFT_FFT_BASE_HPP

#include <shafft/shafft_config.h>
#include <shafft/shafft_types.hpp>

#include <cstddef>

#if SHAFFT_BACKEND_SM100
#include <cuda_runtime_api.h>
#endif

namespace shafft {

class FFT {
public:
  virtual ~FFT() noexcept = default;
  virtual void release() noexcept = 0;
  [[nodiscard]] virtual int setBuffersRaw(void* data, void* work) noexcept = 0;
  [[nodiscard]] virtual int getBuffersRaw(void** data, void** work) noexcept = 0;
  [[nodiscard]] virtual int plan() noexcept = 0;
  [[nodiscard]] virtual int execute(FFTDirection direction) noexcept = 0;
  [[nodiscard]] virtual int normalize() noexcept = 0;
  [[nodiscard]] virtual size_t allocSize() const noexcept = 0;
  [[nodiscard]] virtual size_t globalSize() const noexcept = 0;
  [[nodiscard]] virtual int ndim() const noexcept = 0;
  explicit operator bool() const noexcept { return isConfigured(); }
  [[nodiscard]] virtual bool isActive() const noexcept = 0;
  [[nodiscard]] virtual FFTType fftType() const noexcept = 0;
  [[nodiscard]] PlanState state() const noexcept { return state_; }
  [[nodiscard]] bool isConfigured() const noexcept { return state_ >= PlanState::CONFIGURED; }
  [[nodiscard]] bool isPlanned() const noexcept { return state_ == PlanState::PLANNED; }
#if SHAFFT_BACKEND_SM100
  [[nodiscard]] virtual int setStream(cudaStream_t stream) noexcept = 0;
#endif
  FFT(const FFT&) = delete;
  FFT& operator=(const FFT&) = delete;

protected:
  PlanState state_ = PlanState::UNINITIALIZED;
  FFT() noexcept = default;
  FFT(FFT&&) noexcept = default;
  FFT& operator=(FFT&&) noexcept = default;
};

}  // namespace shafft

#endif  // SHAFFT_FFT_BASE_HPP
