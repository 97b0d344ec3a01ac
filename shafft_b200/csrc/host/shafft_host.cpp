// Host side of SHAFFT on the B200 backend: the FFTND / FFT1D plan objects,
// the free functions of the C++ API, the C ABI and the thread-local error
// state.  Compute is delegated to libshafft_sm100.so through its C ABI
// (include/shafft_sm100.h); this file never touches device memory itself.
//
// Behaviour follows the reference (paths relative to the SHAFFT project):
//   plan state machine             src/cpp/shafft.cpp:26-75, 172-194, 913-983
//   ND configure / validation      src/cpp/shafft_internal.cpp:229-333
//   ND execute (buffer swap, k++)  src/cpp/shafft_internal.cpp:62-127
//   ND normalize (1/sqrt(N))^k     src/cpp/shafft_internal.cpp:129-188
//   1-D execute / normalize        src/cpp/shafft_internal.cpp:584-643,
//                                  src/cpp/fft/hipfft_method/fft1d_method.hip:652-679
//   set/get buffers, queries       src/cpp/shafft_internal.cpp:402-545
//   error state                    src/cpp/shafft_error.cpp:9-162
//   C ABI wrappers                 src/c/shafftc.cpp:60-555
//   config objects                 src/cpp/config_info.cpp:200-711
// With one rank the slab decomposition has no exchange stage, so every
// layout query answers "the whole tensor, offset 0".
#include <shafft/shafft.hpp>
#include <shafft/shafft_error.hpp>
#include <shafft_sm100.h>

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <string>
#include <utility>

namespace {

thread_local int tStatus = 0;
thread_local int tSource = SHAFFT_ERRSRC_NONE;
thread_local int tCode = 0;
thread_local char tMsg[512] = "";

int fail(int status, int source = SHAFFT_ERRSRC_NONE, int code = 0, const char* fmt = nullptr, ...) {
  tStatus = status;
  tSource = source;
  tCode = code;
  tMsg[0] = 0;
  if (fmt) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(tMsg, sizeof(tMsg), fmt, ap);
    va_end(ap);
  }
  return status;
}

int ok() {
  return 0;
}

int st(shafft::Status s) { return static_cast<int>(s); }

// Map a libshafft_sm100 return code onto the SHAFFT status / source pair.
int backend_fail(int rc, const char* what) {
  const char* m = shafft_sm100_last_error_message();
  switch (rc) {
    case SHAFFT_SM100_EALLOC:
      return fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_HIP, shafft_sm100_last_cuda_error(), "%s: %s",
                  what, m);
    case SHAFFT_SM100_ECUDA:
      return fail(SHAFFT_ERR_BACKEND, SHAFFT_ERRSRC_HIP, shafft_sm100_last_cuda_error(), "%s: %s",
                  what, m);
    default:
      return fail(SHAFFT_ERR_BACKEND, SHAFFT_ERRSRC_HIPFFT, rc, "%s: %s", what, m);
  }
}

// Diagnostics on stderr, switched on by SHAFFT_FFT_DIAG=1 as in the
// reference (src/cpp/fft/common/diag.hpp:17-46): one line per plan, execute
// and normalize, tagged [SHAFFT:<module>][r<rank>][<location>].
bool diag_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("SHAFFT_FFT_DIAG");
    return e && e[0] == '1';
  }();
  return on;
}

void diag(const char* module, MPI_Comm comm, const char* location, const char* fmt, ...) {
  if (!diag_enabled()) return;
  int r = -1;
  if (comm != MPI_COMM_NULL) MPI_Comm_rank(comm, &r);
  char line[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(line, sizeof(line), fmt, ap);
  va_end(ap);
  if (r >= 0)
    std::fprintf(stderr, "[SHAFFT:%s][r%d][%s] %s\n", module, r, location, line);
  else
    std::fprintf(stderr, "[SHAFFT:%s][r?][%s] %s\n", module, location, line);
}

}  // namespace

namespace shafft::detail {

// Common state of N-D and 1-D plans.
class PlanBase {
public:
  explicit PlanBase(PlanType t) : type(t) {}
  virtual ~PlanBase() { release(); }

  PlanType type;
  FFTType precision = FFTType::C2C;
  bool configured = false;
  bool planned = false;
  bool active = false;
  MPI_Comm comm = MPI_COMM_NULL;  // dup of the caller's communicator
  void* data = nullptr;           // holds the latest result
  void* work = nullptr;
  int normExp = 0;                // executes since the last normalize
  cudaStream_t stream = nullptr;
  shafft_sm100_plan kplan = nullptr;
  int layoutState = 0;            // 0 = initial, 1 = after a forward transform

  virtual size_t globalSize() const = 0;
  virtual size_t allocSize() const = 0;
  virtual int ndim() const = 0;
  virtual double normFactor(int exponent) const = 0;
  virtual int createBackend() = 0;

  bool isConfigured() const { return configured; }
  bool isPlanned() const { return planned; }
  bool isActive() const { return active; }
  int prec() const { return precision == FFTType::Z2Z ? 1 : 0; }

  void release() {
    if (kplan) {
      shafft_sm100_plan_destroy(kplan);
      kplan = nullptr;
    }
    if (comm != MPI_COMM_NULL) {
      MPI_Comm_free(&comm);
      comm = MPI_COMM_NULL;
    }
    configured = planned = active = false;
    data = work = nullptr;
    normExp = 0;
    layoutState = 0;
  }

  int execute(FFTDirection dir, bool normalized) {
    if (!planned) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (!active) return ok();
    if (!data || !work) return fail(SHAFFT_ERR_NO_BUFFER);
    if (!kplan) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    const double scale = normalized ? normFactor(normExp + 1) : 1.0;
    diag(diagModule(), comm, type == PlanType::PLAN_ND ? "fftndExecute" : "fft1dExecute",
         "begin %s launches=%d src=%p dst=%p scale=%.17g stream=%p",
         dir == FFTDirection::FORWARD ? "FORWARD" : "BACKWARD", shafft_sm100_plan_launches(kplan), data,
         work, scale, (void*)stream);
    int rc = shafft_sm100_execute(kplan, data, work, dir == FFTDirection::FORWARD ? 0 : 1, scale,
                                  stream);
    if (rc) return backend_fail(rc, "execute");
    rc = shafft_sm100_stream_sync(stream);
    if (rc) return backend_fail(rc, "stream synchronize");
    rc = shafft_sm100_plan_status(kplan);
    if (rc) return backend_fail(rc, "execute");
    std::swap(data, work);
    normExp = normalized ? 0 : normExp + 1;
    layoutState = (dir == FFTDirection::FORWARD) ? 1 : 0;
    diag(diagModule(), comm, type == PlanType::PLAN_ND ? "fftndExecute" : "fft1dExecute",
         "end result in data=%p pending normalize exponent=%d", data, normExp);
    return ok();
  }

  int normalize() {
    if (!planned) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (!active) return ok();
    if (!data) return fail(SHAFFT_ERR_NO_BUFFER);
    const double f = normFactor(normExp);
    diag(diagModule(), comm, "normalize", "exponent=%d factor=%.17g data=%p", normExp, f, data);
    if (f != 1.0) {
      int rc = shafft_sm100_scale(data, allocSize(), prec(), f, stream);
      if (rc) return backend_fail(rc, "normalize");
      rc = shafft_sm100_stream_sync(stream);
      if (rc) return backend_fail(rc, "stream synchronize");
    }
    normExp = 0;
    return ok();
  }

  int setBuffers(void* d, void* w) {
    if (!configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (!active || allocSize() == 0) {
      data = work = nullptr;
      return ok();
    }
    if (!d || !w) return fail(SHAFFT_ERR_NULLPTR);
    data = d;
    work = w;
    return ok();
  }

  int getBuffers(void** d, void** w) {
    if (!configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (!d || !w) return fail(SHAFFT_ERR_NULLPTR);
    *d = data;
    *w = work;
    if (active && allocSize() != 0 && (!data || !work)) return fail(SHAFFT_ERR_NO_BUFFER);
    return ok();
  }

  int setStream(cudaStream_t s) {
    if (!configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    stream = s;
    if (kplan) shafft_sm100_set_stream(kplan, s);
    return ok();
  }

  const char* diagModule() const { return type == PlanType::PLAN_ND ? "ND-sm100" : "1D-sm100"; }

  int plan() {
    if (!configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (planned) return fail(SHAFFT_ERR_INVALID_STATE);
    if (active) {
      int rc = createBackend();
      if (rc) return rc;
      if (diag_enabled()) {
        char desc[768] = "";
        shafft_sm100_plan_describe(kplan, desc, sizeof(desc));
        diag(diagModule(), comm, type == PlanType::PLAN_ND ? "fftndPlan" : "fft1dPlan",
             "ndim=%d precision=%s elements=%zu launches=%d passes=%d device_bytes=%zu plan=%s",
             ndim(), prec() ? "Z2Z(double)" : "C2C(float)", globalSize(),
             shafft_sm100_plan_launches(kplan), shafft_sm100_plan_passes(kplan),
             shafft_sm100_plan_device_bytes(kplan), desc);
      }
    }
    planned = true;
    return ok();
  }

  // valid from init on: the plan holds its communicator from configure
  // (src/cpp/detail/plan_data_base.hpp:82-83; src/cpp/shafft.cpp:877-892)
  int communicator(MPI_Comm* out) const {
    if (!out) return fail(SHAFFT_ERR_NULLPTR);
    if (!configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
    if (!active || comm == MPI_COMM_NULL) {
      *out = MPI_COMM_NULL;
      return ok();
    }
    int rc = MPI_Comm_dup(comm, out);
    if (rc != MPI_SUCCESS) return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
    return ok();
  }

protected:
  int bindComm(MPI_Comm c) {
    int rc = MPI_Comm_dup(c, &comm);
    if (rc != MPI_SUCCESS) return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
    int size = 0;
    MPI_Comm_size(comm, &size);
    if (size != 1) {
      MPI_Comm_free(&comm);
      comm = MPI_COMM_NULL;
      return fail(SHAFFT_ERR_INVALID_COMM, SHAFFT_ERRSRC_NONE, size,
                  "the sm100 backend runs one rank per plan (communicator size %d)", size);
    }
    return ok();
  }
};

struct FFTNDPlan : PlanBase {
  FFTNDPlan() : PlanBase(PlanType::PLAN_ND) {}
  std::vector<size_t> dims;
  TransformLayout policy = TransformLayout::REDISTRIBUTED;
  long double normDen = 1.0L;

  size_t globalSize() const override {
    size_t n = 1;
    for (size_t d : dims) n *= d;
    return dims.empty() ? 0 : n;
  }
  size_t allocSize() const override { return active ? globalSize() : 0; }
  int ndim() const override { return (int)dims.size(); }
  double normFactor(int k) const override {
    long double f = 1.0L / std::pow(normDen, (long double)k);
    return precision == FFTType::C2C ? (double)(float)f : (double)f;
  }
  int createBackend() override {
    std::vector<int64_t> d(dims.begin(), dims.end());
    int rc = shafft_sm100_plan_create_nd(&kplan, (int)d.size(), d.data(), prec());
    if (rc) {
      kplan = nullptr;
      return backend_fail(rc, "plan");
    }
    shafft_sm100_set_stream(kplan, stream);
    return ok();
  }

  int configure(int nd, const int* commDims, const int* dimensions, FFTType p, MPI_Comm c,
                TransformLayout pol) {
    if (configured) return fail(SHAFFT_ERR_INVALID_STATE);
    if (c == MPI_COMM_NULL) {  // inactive rank
      configured = true;
      active = false;
      precision = p;
      return ok();
    }
    if (!commDims || !dimensions) return fail(SHAFFT_ERR_NULLPTR);
    if (nd <= 0) return fail(SHAFFT_ERR_INVALID_DIM);
    for (int i = 0; i < nd; ++i)
      if (dimensions[i] < 1) return fail(SHAFFT_ERR_INVALID_DIM);
    if (commDims[nd - 1] != 1) return fail(SHAFFT_ERR_INVALID_DECOMP);
    for (int i = 0; i < nd; ++i)
      if (commDims[i] < 1 || commDims[i] > dimensions[i]) return fail(SHAFFT_ERR_INVALID_DECOMP);
    long long grid = 1;
    for (int i = 0; i < nd; ++i) grid *= commDims[i];
    if (p != FFTType::C2C && p != FFTType::Z2Z) return fail(SHAFFT_ERR_INVALID_FFTTYPE);
    int size = 1;
    if (MPI_Comm_size(c, &size) != MPI_SUCCESS) return fail(SHAFFT_ERR_INVALID_COMM);
    if (grid != size)
      return fail(SHAFFT_ERR_INVALID_DECOMP, SHAFFT_ERRSRC_NONE, 0,
                  "process grid of %lld ranks on a communicator of %d", grid, size);
    int rc = bindComm(c);
    if (rc) return rc;
    precision = p;
    policy = pol;
    dims.assign(dimensions, dimensions + nd);
    long double n = 1.0L;
    for (size_t d : dims) n *= (long double)d;
    normDen = std::sqrt(n);
    active = true;
    configured = true;
    return ok();
  }
};

struct FFT1DPlan : PlanBase {
  FFT1DPlan() : PlanBase(PlanType::PLAN_1D) {}
  size_t N = 0;

  size_t globalSize() const override { return N; }
  size_t allocSize() const override { return active ? N : 0; }
  int ndim() const override { return 1; }
  double normFactor(int k) const override {
    if (precision == FFTType::C2C)
      return (double)(1.0f / std::pow(std::sqrt((float)N), (float)k));
    return 1.0 / std::pow(std::sqrt((double)N), (double)k);
  }
  int createBackend() override {
    int rc = shafft_sm100_plan_create_1d(&kplan, (int64_t)N, prec());
    if (rc) {
      kplan = nullptr;
      return backend_fail(rc, "plan");
    }
    shafft_sm100_set_stream(kplan, stream);
    return ok();
  }
  int configure(size_t globalN, FFTType p, MPI_Comm c) {
    if (configured) return fail(SHAFFT_ERR_INVALID_STATE);
    if (c == MPI_COMM_NULL) {
      configured = true;
      active = false;
      precision = p;
      return ok();
    }
    if (p != FFTType::C2C && p != FFTType::Z2Z) return fail(SHAFFT_ERR_INVALID_FFTTYPE);
    if (globalN == 0) return fail(SHAFFT_ERR_INVALID_DIM);
    if (globalN > (size_t)INT_MAX) return fail(SHAFFT_ERR_SIZE_OVERFLOW);
    int rc = bindComm(c);
    if (rc) return rc;
    precision = p;
    N = globalN;
    active = true;
    configured = true;
    return ok();
  }
};

}  // namespace shafft::detail

using shafft::detail::FFT1DPlan;
using shafft::detail::FFTNDPlan;
using shafft::detail::PlanBase;

namespace {

PlanBase* asPlan(void* p) { return static_cast<PlanBase*>(p); }

int fillLayout(const PlanBase* p, size_t* subsize, size_t* offset) {
  if (p->type == shafft::PlanType::PLAN_ND) {
    const auto* nd = static_cast<const FFTNDPlan*>(p);
    for (size_t i = 0; i < nd->dims.size(); ++i) {
      subsize[i] = p->active ? nd->dims[i] : 0;
      offset[i] = 0;
    }
  } else {
    const auto* od = static_cast<const FFT1DPlan*>(p);
    subsize[0] = p->active ? od->N : 0;
    offset[0] = 0;
  }
  return ok();
}

// contiguous axes: ND -> all axes (nda = 0); 1-D -> none, the one axis is
// the distributed one (reference src/cpp/shafft.cpp FFT1D::getAxes comment)
int ncaOf(const PlanBase* p) { return p->type == shafft::PlanType::PLAN_ND ? p->ndim() : 0; }
int ndaOf(const PlanBase* p) { return p->type == shafft::PlanType::PLAN_ND ? 0 : 1; }

int fillAxes(const PlanBase* p, int* ca, int* da) {
  const int nca = ncaOf(p), nda = ndaOf(p);
  if ((nca && !ca) || (nda && !da)) return fail(SHAFFT_ERR_NULLPTR);
  for (int i = 0; i < nca; ++i) ca[i] = i;
  for (int i = 0; i < nda; ++i) da[i] = i;
  return ok();
}

char* dupString(const char* s, size_t* len) {
  size_t n = strlen(s);
  char* r = (char*)malloc(n + 1);
  if (r) memcpy(r, s, n + 1);
  if (len) *len = r ? n : 0;
  return r;
}

void hostAndDevice(char** host, size_t* hostLen, char** dev, size_t* devLen) {
  char hn[256] = "localhost";
  gethostname(hn, sizeof(hn) - 1);
  *host = dupString(hn, hostLen);
  char dn[256] = "";
  if (shafft_sm100_device_name(dn, sizeof(dn)) == 0 && dn[0]) {
    *dev = dupString(dn, devLen);
  } else {
    *dev = nullptr;
    *devLen = 0;
  }
}

}  // namespace

// ===========================================================================
// C++ API
// ===========================================================================
namespace shafft {

FFTND::~FFTND() noexcept { release(); }

void FFTND::release() noexcept {
  delete data_;
  data_ = nullptr;
  state_ = PlanState::UNINITIALIZED;
}

FFTND::FFTND(FFTND&& o) noexcept : data_(o.data_) {
  state_ = o.state_;
  o.data_ = nullptr;
  o.state_ = PlanState::UNINITIALIZED;
}

FFTND& FFTND::operator=(FFTND&& o) noexcept {
  if (this != &o) {
    delete data_;
    data_ = o.data_;
    state_ = o.state_;
    o.data_ = nullptr;
    o.state_ = PlanState::UNINITIALIZED;
  }
  return *this;
}

int FFTND::init(const std::vector<int>& commDims, const std::vector<size_t>& dimensions, FFTType type,
                MPI_Comm comm, TransformLayout output) noexcept {
  try {
    if (state_ != PlanState::UNINITIALIZED) return fail(SHAFFT_ERR_INVALID_STATE);
    if (commDims.size() != dimensions.size()) return fail(SHAFFT_ERR_DIM_MISMATCH);
    std::vector<int> d(dimensions.size());
    for (size_t i = 0; i < dimensions.size(); ++i) {
      if (dimensions[i] > (size_t)INT_MAX) return fail(SHAFFT_ERR_SIZE_OVERFLOW);
      d[i] = (int)dimensions[i];
    }
    auto* p = new FFTNDPlan();
    int rc = p->configure((int)d.size(), commDims.data(), d.data(), type, comm, output);
    if (rc) {
      delete p;
      return rc;
    }
    data_ = p;
    state_ = PlanState::CONFIGURED;
    return ok();
  } catch (...) {
    return fail(st(err::mapExceptionToStatus()), SHAFFT_ERRSRC_SYSTEM);
  }
}

int FFTND::init(shafft_nd_config_t& cfg) noexcept {
  if (!(cfg.flags & SHAFFT_CONFIG_RESOLVED)) {
    int rc = shafftConfigNDResolve(&cfg);
    if (rc) return rc;
  }
  std::vector<int> cd(cfg.commDims, cfg.commDims + cfg.ndim);
  std::vector<size_t> dims(cfg.globalShape, cfg.globalShape + cfg.ndim);
  return init(cd, dims, cfg.precision == SHAFFT_Z2Z ? FFTType::Z2Z : FFTType::C2C, cfg.worldComm,
              cfg.outputPolicy == SHAFFT_LAYOUT_INITIAL ? TransformLayout::INITIAL
                                                        : TransformLayout::REDISTRIBUTED);
}

int FFTND::plan() noexcept {
  if (state_ != PlanState::CONFIGURED) {
    if (state_ == PlanState::PLANNED) return fail(SHAFFT_ERR_INVALID_STATE);
    return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  }
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  int rc = data_->plan();
  if (rc) return rc;
  state_ = PlanState::PLANNED;
  return ok();
}

int FFTND::setBuffers(complexf* d, complexf* w) noexcept { return setBuffersRaw(d, w); }
int FFTND::setBuffers(complexd* d, complexd* w) noexcept { return setBuffersRaw(d, w); }
int FFTND::setBuffers(cuFloatComplex* d, cuFloatComplex* w) noexcept { return setBuffersRaw(d, w); }
int FFTND::setBuffers(cuDoubleComplex* d, cuDoubleComplex* w) noexcept { return setBuffersRaw(d, w); }
int FFTND::getBuffers(complexf** d, complexf** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFTND::getBuffers(complexd** d, complexd** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFTND::getBuffers(cuFloatComplex** d, cuFloatComplex** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFTND::getBuffers(cuDoubleComplex** d, cuDoubleComplex** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFTND::setBuffersRaw(void* d, void* w) noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->setBuffers(d, w);
}
int FFTND::getBuffersRaw(void** d, void** w) noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->getBuffers(d, w);
}
int FFTND::execute(FFTDirection dir) noexcept {
  if (state_ != PlanState::PLANNED || !data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->execute(dir, false);
}
int FFTND::executeNormalized(FFTDirection dir) noexcept {
  if (state_ != PlanState::PLANNED || !data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->execute(dir, true);
}
int FFTND::normalize() noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->normalize();
}
size_t FFTND::allocSize() const noexcept { return data_ ? data_->allocSize() : 0; }
size_t FFTND::globalSize() const noexcept { return data_ ? data_->globalSize() : 0; }
int FFTND::ndim() const noexcept { return data_ ? data_->ndim() : 0; }
FFTType FFTND::fftType() const noexcept { return data_ ? data_->precision : FFTType::C2C; }
bool FFTND::isActive() const noexcept { return data_ && data_->isActive(); }
int FFTND::getLayout(std::vector<size_t>& subsize, std::vector<size_t>& offset,
                     TensorLayout) const noexcept {
  if (!data_ || !data_->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  subsize.resize(data_->ndim());
  offset.resize(data_->ndim());
  return fillLayout(data_, subsize.data(), offset.data());
}
int FFTND::getAxes(std::vector<int>& ca, std::vector<int>& da, TensorLayout) const noexcept {
  if (!data_ || !data_->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  ca.resize(ncaOf(data_));
  da.resize(ndaOf(data_));
  return fillAxes(data_, ca.data(), da.data());
}
int FFTND::setStream(cudaStream_t s) noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->setStream(s);
}
int FFTND::getCommunicator(MPI_Comm* out) const noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->communicator(out);
}

FFT1D::~FFT1D() noexcept { release(); }
void FFT1D::release() noexcept {
  delete data_;
  data_ = nullptr;
  state_ = PlanState::UNINITIALIZED;
}
FFT1D::FFT1D(FFT1D&& o) noexcept : data_(o.data_) {
  state_ = o.state_;
  o.data_ = nullptr;
  o.state_ = PlanState::UNINITIALIZED;
}
FFT1D& FFT1D::operator=(FFT1D&& o) noexcept {
  if (this != &o) {
    release();
    data_ = o.data_;
    state_ = o.state_;
    o.data_ = nullptr;
    o.state_ = PlanState::UNINITIALIZED;
  }
  return *this;
}
int FFT1D::init(size_t globalN, size_t, size_t, FFTType precision, MPI_Comm comm) noexcept {
  try {
    if (state_ != PlanState::UNINITIALIZED) return fail(SHAFFT_ERR_INVALID_STATE);
    auto* p = new FFT1DPlan();
    int rc = p->configure(globalN, precision, comm);
    if (rc) {
      delete p;
      return rc;
    }
    data_ = p;
    state_ = PlanState::CONFIGURED;
    return ok();
  } catch (...) {
    return fail(st(err::mapExceptionToStatus()), SHAFFT_ERRSRC_SYSTEM);
  }
}
int FFT1D::init(shafft_1d_config_t& cfg) noexcept {
  if (!(cfg.flags & SHAFFT_CONFIG_RESOLVED)) {
    int rc = shafftConfig1DResolve(&cfg);
    if (rc) return rc;
  }
  return init(cfg.globalSize, cfg.initial.localSize, cfg.initial.localStart,
              cfg.precision == SHAFFT_Z2Z ? FFTType::Z2Z : FFTType::C2C, cfg.worldComm);
}
int FFT1D::plan() noexcept {
  if (state_ != PlanState::CONFIGURED || !data_) return fail(SHAFFT_ERR_INVALID_STATE);
  int rc = data_->plan();
  if (rc) return rc;
  state_ = PlanState::PLANNED;
  return ok();
}
int FFT1D::setBuffers(complexf* d, complexf* w) noexcept { return setBuffersRaw(d, w); }
int FFT1D::setBuffers(complexd* d, complexd* w) noexcept { return setBuffersRaw(d, w); }
int FFT1D::setBuffers(cuFloatComplex* d, cuFloatComplex* w) noexcept { return setBuffersRaw(d, w); }
int FFT1D::setBuffers(cuDoubleComplex* d, cuDoubleComplex* w) noexcept { return setBuffersRaw(d, w); }
int FFT1D::getBuffers(complexf** d, complexf** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFT1D::getBuffers(complexd** d, complexd** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFT1D::getBuffers(cuFloatComplex** d, cuFloatComplex** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFT1D::getBuffers(cuDoubleComplex** d, cuDoubleComplex** w) noexcept {
  return getBuffersRaw(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w));
}
int FFT1D::setBuffersRaw(void* d, void* w) noexcept {
  if (!data_) return fail(SHAFFT_ERR_NULLPTR);
  return data_->setBuffers(d, w);
}
int FFT1D::getBuffersRaw(void** d, void** w) noexcept {
  if (!data_) return fail(SHAFFT_ERR_NULLPTR);
  return data_->getBuffers(d, w);
}
int FFT1D::execute(FFTDirection dir) noexcept {
  if (state_ != PlanState::PLANNED || !data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->execute(dir, false);
}
int FFT1D::executeNormalized(FFTDirection dir) noexcept {
  if (state_ != PlanState::PLANNED || !data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->execute(dir, true);
}
int FFT1D::normalize() noexcept {
  if (!data_) return fail(SHAFFT_ERR_NULLPTR);
  return data_->normalize();
}
std::vector<size_t> FFT1D::globalShape() const noexcept {
  if (!data_ || !data_->configured) return {};
  return {data_->globalSize()};
}
size_t FFT1D::globalSize() const noexcept { return data_ ? data_->globalSize() : 0; }
size_t FFT1D::localSize() const noexcept { return data_ ? data_->allocSize() : 0; }
size_t FFT1D::allocSize() const noexcept { return data_ ? data_->allocSize() : 0; }
int FFT1D::ndim() const noexcept { return 1; }
FFTType FFT1D::fftType() const noexcept { return data_ ? data_->precision : FFTType::C2C; }
bool FFT1D::isActive() const noexcept { return data_ && data_->configured && data_->isActive(); }
int FFT1D::getLayout(std::vector<size_t>& localShape, std::vector<size_t>& offset,
                     TensorLayout) const noexcept {
  if (!data_ || !data_->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  localShape.assign(1, 0);
  offset.assign(1, 0);
  return fillLayout(data_, localShape.data(), offset.data());
}
int FFT1D::getAxes(std::vector<int>& ca, std::vector<int>& da, TensorLayout) const noexcept {
  if (!data_ || !data_->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  ca.resize(ncaOf(data_));
  da.resize(ndaOf(data_));
  return fillAxes(data_, ca.data(), da.data());
}
int FFT1D::setStream(cudaStream_t s) noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->setStream(s);
}
int FFT1D::getCommunicator(MPI_Comm* out) const noexcept {
  if (!data_) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return data_->communicator(out);
}

// ---- free functions --------------------------------------------------------

int setStream(detail::PlanBase* plan, cudaStream_t s) {
  if (!plan) return fail(SHAFFT_ERR_NULLPTR);
  return plan->setStream(s);
}
int setBuffers(detail::PlanBase* p, cuFloatComplex* d, cuFloatComplex* w) noexcept {
  return p ? p->setBuffers(d, w) : fail(SHAFFT_ERR_NULLPTR);
}
int setBuffers(detail::PlanBase* p, cuDoubleComplex* d, cuDoubleComplex* w) noexcept {
  return p ? p->setBuffers(d, w) : fail(SHAFFT_ERR_NULLPTR);
}
int setBuffers(detail::PlanBase* p, complexf* d, complexf* w) noexcept {
  return p ? p->setBuffers(d, w) : fail(SHAFFT_ERR_NULLPTR);
}
int setBuffers(detail::PlanBase* p, complexd* d, complexd* w) noexcept {
  return p ? p->setBuffers(d, w) : fail(SHAFFT_ERR_NULLPTR);
}
int getBuffers(detail::PlanBase* p, cuFloatComplex** d, cuFloatComplex** w) noexcept {
  return p ? p->getBuffers(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w))
           : fail(SHAFFT_ERR_NULLPTR);
}
int getBuffers(detail::PlanBase* p, cuDoubleComplex** d, cuDoubleComplex** w) noexcept {
  return p ? p->getBuffers(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w))
           : fail(SHAFFT_ERR_NULLPTR);
}
int getBuffers(detail::PlanBase* p, complexf** d, complexf** w) noexcept {
  return p ? p->getBuffers(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w))
           : fail(SHAFFT_ERR_NULLPTR);
}
int getBuffers(detail::PlanBase* p, complexd** d, complexd** w) noexcept {
  return p ? p->getBuffers(reinterpret_cast<void**>(d), reinterpret_cast<void**>(w))
           : fail(SHAFFT_ERR_NULLPTR);
}

int allocBuffer(size_t count, complexf** buf) noexcept {
  return shafftAllocBufferF(count, reinterpret_cast<void**>(buf));
}
int allocBuffer(size_t count, complexd** buf) noexcept {
  return shafftAllocBufferD(count, reinterpret_cast<void**>(buf));
}
int freeBuffer(complexf* buf) noexcept { return shafftFreeBufferF(buf); }
int freeBuffer(complexd* buf) noexcept { return shafftFreeBufferD(buf); }
int copyToBuffer(complexf* dst, const complexf* src, size_t count) noexcept {
  return shafftCopyToBufferF(dst, src, count);
}
int copyToBuffer(complexd* dst, const complexd* src, size_t count) noexcept {
  return shafftCopyToBufferD(dst, src, count);
}
int copyFromBuffer(complexf* dst, const complexf* src, size_t count) noexcept {
  return shafftCopyFromBufferF(dst, src, count);
}
int copyFromBuffer(complexd* dst, const complexd* src, size_t count) noexcept {
  return shafftCopyFromBufferD(dst, src, count);
}

int planNDCreate(detail::FFTNDPlan** out) {
  if (!out) return fail(SHAFFT_ERR_NULLPTR);
  *out = new (std::nothrow) detail::FFTNDPlan();
  return *out ? ok() : fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_SYSTEM);
}
int FFT1DCreate(detail::FFT1DPlan** out) {
  if (!out) return fail(SHAFFT_ERR_NULLPTR);
  *out = new (std::nothrow) detail::FFT1DPlan();
  return *out ? ok() : fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_SYSTEM);
}

int configurationND(const std::vector<size_t>& size, FFTType precision, std::vector<int>& commDims,
                    int& nda, std::vector<size_t>& subsize, std::vector<size_t>& offset,
                    int& commSize, DecompositionStrategy strategy, size_t memLimit, MPI_Comm comm) {
  const int ndim = (int)size.size();
  if ((int)subsize.size() != ndim || (int)offset.size() != ndim || (int)commDims.size() != ndim)
    return fail(SHAFFT_ERR_DIM_MISMATCH);
  std::vector<int> isz(ndim);
  for (int i = 0; i < ndim; ++i) {
    if (size[i] > (size_t)INT_MAX) return fail(SHAFFT_ERR_SIZE_OVERFLOW);
    isz[i] = (int)size[i];
  }
  return shafftConfigurationND(ndim, isz.data(), precision == FFTType::Z2Z ? SHAFFT_Z2Z : SHAFFT_C2C,
                               commDims.data(), &nda, subsize.data(), offset.data(), &commSize,
                               strategy == DecompositionStrategy::MINIMIZE_NDA ? SHAFFT_MINIMIZE_NDA
                                                                               : SHAFFT_MAXIMIZE_NDA,
                               memLimit, comm);
}

int configuration1D(size_t globalN, size_t& localN, size_t& localStart, FFTType precision,
                    MPI_Comm comm) {
  size_t alloc = 0;
  return shafftConfiguration1D(globalN, &localN, &localStart, &alloc,
                               precision == FFTType::Z2Z ? SHAFFT_Z2Z : SHAFFT_C2C, comm);
}

int planND(detail::FFTNDPlan* plan, const std::vector<int>& commDims,
           const std::vector<size_t>& dimensions, FFTType precision, MPI_Comm comm) {
  if (!plan) return fail(SHAFFT_ERR_NULLPTR);
  if (commDims.size() != dimensions.size()) return fail(SHAFFT_ERR_DIM_MISMATCH);
  std::vector<int> d(dimensions.size());
  for (size_t i = 0; i < dimensions.size(); ++i) {
    if (dimensions[i] > (size_t)INT_MAX) return fail(SHAFFT_ERR_SIZE_OVERFLOW);
    d[i] = (int)dimensions[i];
  }
  return plan->configure((int)d.size(), commDims.data(), d.data(), precision, comm,
                         TransformLayout::REDISTRIBUTED);
}

int destroy(detail::PlanBase** plan) {
  if (!plan || !*plan) return fail(SHAFFT_ERR_NULLPTR);
  delete *plan;
  *plan = nullptr;
  return ok();
}

int getLayout(const detail::PlanBase* plan, std::vector<size_t>& subsize,
              std::vector<size_t>& offset, TensorLayout) {
  if (!plan || !plan->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  subsize.resize(plan->ndim());
  offset.resize(plan->ndim());
  return fillLayout(plan, subsize.data(), offset.data());
}

int getAxes(const detail::PlanBase* plan, std::vector<int>& ca, std::vector<int>& da, TensorLayout) {
  if (!plan || !plan->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  ca.resize(ncaOf(plan));
  da.resize(ndaOf(plan));
  return fillAxes(plan, ca.data(), da.data());
}

int getAllocSize(const detail::PlanBase* plan, size_t& localAllocSize) {
  if (!plan || !plan->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  localAllocSize = plan->allocSize();
  return ok();
}

int execute(detail::PlanBase* plan, FFTDirection direction) {
  if (!plan) return fail(SHAFFT_ERR_NULLPTR);
  return plan->execute(direction, false);
}

int normalize(detail::PlanBase* plan) {
  if (!plan) return fail(SHAFFT_ERR_NULLPTR);
  if (!plan->planned) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return plan->normalize();
}

int finalize() noexcept { return shafftFinalize(); }

ConfigND::ConfigND(const std::vector<size_t>& globalShape, FFTType precision,
                   const std::vector<int>& commDims, int hintNda, DecompositionStrategy strategy,
                   TransformLayout outputPolicy, size_t memLimit, MPI_Comm comm) noexcept {
  const int nd = (int)globalShape.size();
  status_ = shafftConfigNDInit(
      &cfg_, nd, globalShape.data(), precision == FFTType::Z2Z ? SHAFFT_Z2Z : SHAFFT_C2C,
      commDims.size() == (size_t)nd ? commDims.data() : nullptr, hintNda,
      strategy == DecompositionStrategy::MINIMIZE_NDA ? SHAFFT_MINIMIZE_NDA : SHAFFT_MAXIMIZE_NDA,
      outputPolicy == TransformLayout::INITIAL ? SHAFFT_LAYOUT_INITIAL : SHAFFT_LAYOUT_REDISTRIBUTED,
      memLimit, comm);
}
ConfigND::ConfigND(ConfigND&& o) noexcept : cfg_(o.cfg_), status_(o.status_) {
  memset(&o.cfg_, 0, sizeof(o.cfg_));
  o.status_ = -1;
}
ConfigND& ConfigND::operator=(ConfigND&& o) noexcept {
  if (this != &o) {
    shafftConfigNDRelease(&cfg_);
    cfg_ = o.cfg_;
    status_ = o.status_;
    memset(&o.cfg_, 0, sizeof(o.cfg_));
    o.status_ = -1;
  }
  return *this;
}
ConfigND::~ConfigND() noexcept { shafftConfigNDRelease(&cfg_); }
int ConfigND::resolve() noexcept { return status_ = shafftConfigNDResolve(&cfg_); }

Config1D::Config1D(size_t globalSize, FFTType precision, MPI_Comm comm) noexcept {
  status_ = shafftConfig1DInit(&cfg_, globalSize, precision == FFTType::Z2Z ? SHAFFT_Z2Z : SHAFFT_C2C,
                               comm);
}
Config1D::Config1D(Config1D&& o) noexcept : cfg_(o.cfg_), status_(o.status_) {
  memset(&o.cfg_, 0, sizeof(o.cfg_));
  o.status_ = -1;
}
Config1D& Config1D::operator=(Config1D&& o) noexcept {
  if (this != &o) {
    shafftConfig1DRelease(&cfg_);
    cfg_ = o.cfg_;
    status_ = o.status_;
    memset(&o.cfg_, 0, sizeof(o.cfg_));
    o.status_ = -1;
  }
  return *this;
}
Config1D::~Config1D() noexcept { shafftConfig1DRelease(&cfg_); }
int Config1D::resolve() noexcept { return status_ = shafftConfig1DResolve(&cfg_); }

}  // namespace shafft

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int shafftLastErrorStatus(void) { return tStatus; }
int shafftLastErrorSource(void) { return tSource; }
int shafftLastErrorDomainCode(void) { return tCode; }
void shafftClearLastError(void) {
  tStatus = 0;
  tSource = SHAFFT_ERRSRC_NONE;
  tCode = 0;
  tMsg[0] = 0;
}
const char* shafftErrorSourceName(int source) {
  switch (source) {
    case SHAFFT_ERRSRC_NONE: return "SHAFFT";
    case SHAFFT_ERRSRC_MPI: return "MPI";
    case SHAFFT_ERRSRC_HIP: return "CUDA";
    case SHAFFT_ERRSRC_HIPFFT: return "sm100";
    case SHAFFT_ERRSRC_FFTW: return "FFTW";
    case SHAFFT_ERRSRC_SYSTEM: return "System";
    default: return "Unknown";
  }
}
int shafftLastErrorMessage(char* buf, int buflen) {
  if (!buf || buflen <= 0) return 0;
  buf[0] = 0;
  int n = 0;
  if (tSource == SHAFFT_ERRSRC_MPI && tCode != MPI_SUCCESS) {
    char m[MPI_MAX_ERROR_STRING];
    int len = 0;
    MPI_Error_string(tCode, m, &len);
    n = snprintf(buf, buflen, "%s", m);
  } else if (tMsg[0]) {
    n = snprintf(buf, buflen, "%s", tMsg);
  } else if (tStatus != 0) {
    n = snprintf(buf, buflen, "%s", shafft::err::statusToString(tStatus));
  }
  if (n >= buflen) n = buflen - 1;
  if (n < 0) n = 0;
  return n;
}

int shafftSetStream(void* planPtr, cudaStream_t stream) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  return asPlan(planPtr)->setStream(stream);
}

// ---- config objects --------------------------------------------------------

static void freeLayout(shafft_nd_layout_t* l) {
  free(l->subsize);
  free(l->offset);
  free(l->contiguousAxes);
  free(l->distributedAxes);
  memset(l, 0, sizeof(*l));
}

int shafftConfigNDInit(shafft_nd_config_t* cfg, int ndim, const size_t* globalShape,
                       shafft_t precision, const int* commDims, int hintNda,
                       shafft_decomposition_strategy_t strategy,
                       shafft_transform_layout_t outputPolicy, size_t memLimit, MPI_Comm comm) {
  if (!cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (ndim < 1) return fail(SHAFFT_ERR_INVALID_DIM);
  if (!globalShape) return fail(SHAFFT_ERR_NULLPTR);
  if (cfg->structSize == sizeof(shafft_nd_config_t)) return fail(SHAFFT_ERR_INVALID_STATE);
  memset(cfg, 0, sizeof(*cfg));
  cfg->structSize = sizeof(shafft_nd_config_t);
  cfg->apiVersion = 1;
  cfg->ndim = ndim;
  cfg->activeRank = -1;
  cfg->worldComm = MPI_COMM_NULL;
  cfg->activeComm = MPI_COMM_NULL;
  const size_t n = (size_t)ndim;
  cfg->globalShape = (size_t*)calloc(n, sizeof(size_t));
  cfg->hintCommDims = (int*)calloc(n, sizeof(int));
  cfg->commDims = (int*)calloc(n, sizeof(int));
  shafft_nd_layout_t* ls[2] = {&cfg->initial, &cfg->output};
  for (auto* l : ls) {
    l->subsize = (size_t*)calloc(n, sizeof(size_t));
    l->offset = (size_t*)calloc(n, sizeof(size_t));
    l->contiguousAxes = (int*)calloc(n, sizeof(int));
    l->distributedAxes = (int*)calloc(n, sizeof(int));
  }
  if (!cfg->globalShape || !cfg->hintCommDims || !cfg->commDims || !cfg->initial.subsize ||
      !cfg->initial.offset || !cfg->initial.contiguousAxes || !cfg->initial.distributedAxes ||
      !cfg->output.subsize || !cfg->output.offset || !cfg->output.contiguousAxes ||
      !cfg->output.distributedAxes) {
    shafftConfigNDRelease(cfg);
    return fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_SYSTEM);
  }
  for (int i = 0; i < ndim; ++i) cfg->globalShape[i] = globalShape[i];
  if (commDims)
    for (int i = 0; i < ndim; ++i) cfg->hintCommDims[i] = commDims[i];
  cfg->precision = precision;
  cfg->hintNda = hintNda;
  cfg->strategy = strategy;
  cfg->outputPolicy = outputPolicy;
  cfg->memLimit = memLimit;
  int rc = MPI_Comm_dup(comm, &cfg->worldComm);
  if (rc != MPI_SUCCESS) {
    shafftConfigNDRelease(cfg);
    return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
  }
  rc = shafftConfigNDResolve(cfg);
  if (rc) {
    shafftConfigNDRelease(cfg);
    return rc;
  }
  return ok();
}

void shafftConfigNDRelease(shafft_nd_config_t* cfg) {
  if (!cfg || cfg->structSize == 0) return;
  free(cfg->globalShape);
  free(cfg->hintCommDims);
  free(cfg->commDims);
  freeLayout(&cfg->initial);
  freeLayout(&cfg->output);
  free(cfg->hostname);
  free(cfg->deviceName);
  if (cfg->worldComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->worldComm);
  if (cfg->activeComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->activeComm);
  memset(cfg, 0, sizeof(*cfg));
}

int shafftConfigNDResolve(shafft_nd_config_t* cfg) {
  if (!cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (cfg->structSize != sizeof(shafft_nd_config_t)) return fail(SHAFFT_ERR_INVALID_STATE);
  const int nd = cfg->ndim;
  std::vector<int> isz(nd), cd(nd);
  for (int i = 0; i < nd; ++i) {
    if (cfg->globalShape[i] == 0) return cfg->status = fail(SHAFFT_ERR_INVALID_DIM);
    if (cfg->globalShape[i] > (size_t)INT_MAX) return cfg->status = fail(SHAFFT_ERR_SIZE_OVERFLOW);
    isz[i] = (int)cfg->globalShape[i];
    cd[i] = cfg->hintCommDims[i];
  }
  int nda = cfg->hintNda, commSize = 0;
  std::vector<size_t> sub(nd), off(nd);
  int rc = shafftConfigurationND(nd, isz.data(), cfg->precision, cd.data(), &nda, sub.data(),
                                 off.data(), &commSize, cfg->strategy, cfg->memLimit,
                                 cfg->worldComm);
  if (rc) return cfg->status = rc;
  cfg->flags = 0;
  for (int i = 0; i < nd; ++i) {
    if (cfg->hintCommDims[i] != 0 && cfg->hintCommDims[i] != cd[i])
      cfg->flags |= SHAFFT_CONFIG_CHANGED_COMM_DIMS;
    cfg->commDims[i] = cd[i];
  }
  if (cfg->hintNda != 0 && cfg->hintNda != nda) cfg->flags |= SHAFFT_CONFIG_CHANGED_NDA;
  cfg->nda = nda;
  cfg->commSize = commSize;
  size_t total = 1;
  for (int i = 0; i < nd; ++i) total *= cfg->globalShape[i];
  cfg->allocElements = total;
  shafft_nd_layout_t* ls[2] = {&cfg->initial, &cfg->output};
  for (auto* l : ls) {
    for (int i = 0; i < nd; ++i) {
      l->subsize[i] = sub[i];
      l->offset[i] = off[i];
      l->contiguousAxes[i] = i;
    }
    l->localElements = total;
    l->hasLocalElements = total > 0;
  }
  cfg->isActive = 1;
  cfg->activeRank = 0;
  cfg->activeSize = 1;
  if (cfg->activeComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->activeComm);
  MPI_Comm_dup(cfg->worldComm, &cfg->activeComm);
  cfg->nodeId = 0;
  cfg->nodeCount = 1;
  free(cfg->hostname);
  free(cfg->deviceName);
  hostAndDevice(&cfg->hostname, &cfg->hostnameLen, &cfg->deviceName, &cfg->deviceNameLen);
  cfg->flags |= SHAFFT_CONFIG_RESOLVED;
  cfg->status = 0;
  return ok();
}

int shafftNDInitFromConfig(void* planPtr, shafft_nd_config_t* cfg) {
  if (!planPtr || !cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (!(cfg->flags & SHAFFT_CONFIG_RESOLVED)) {
    int rc = shafftConfigNDResolve(cfg);
    if (rc) return rc;
  }
  std::vector<int> dims(cfg->ndim);
  for (int i = 0; i < cfg->ndim; ++i) dims[i] = (int)cfg->globalShape[i];
  return shafftNDInit(planPtr, cfg->ndim, cfg->commDims, dims.data(), cfg->precision, cfg->worldComm,
                      cfg->outputPolicy);
}

int shafftConfig1DInit(shafft_1d_config_t* cfg, size_t globalSize, shafft_t precision,
                       MPI_Comm comm) {
  if (!cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (globalSize == 0) return fail(SHAFFT_ERR_INVALID_DIM);
  if (cfg->structSize == sizeof(shafft_1d_config_t)) return fail(SHAFFT_ERR_INVALID_STATE);
  memset(cfg, 0, sizeof(*cfg));
  cfg->structSize = sizeof(shafft_1d_config_t);
  cfg->apiVersion = 1;
  cfg->globalSize = globalSize;
  cfg->precision = precision;
  cfg->activeRank = -1;
  int rc = MPI_Comm_dup(comm, &cfg->worldComm);
  if (rc != MPI_SUCCESS) {
    memset(cfg, 0, sizeof(*cfg));
    return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
  }
  rc = shafftConfig1DResolve(cfg);
  if (rc) {
    shafftConfig1DRelease(cfg);
    return rc;
  }
  return ok();
}

void shafftConfig1DRelease(shafft_1d_config_t* cfg) {
  if (!cfg || cfg->structSize == 0) return;
  free(cfg->hostname);
  free(cfg->deviceName);
  if (cfg->worldComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->worldComm);
  if (cfg->activeComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->activeComm);
  memset(cfg, 0, sizeof(*cfg));
}

int shafftConfig1DResolve(shafft_1d_config_t* cfg) {
  if (!cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (cfg->structSize != sizeof(shafft_1d_config_t)) return fail(SHAFFT_ERR_INVALID_STATE);
  size_t ln = 0, ls = 0, as = 0;
  int rc = shafftConfiguration1D(cfg->globalSize, &ln, &ls, &as, cfg->precision, cfg->worldComm);
  if (rc) return cfg->status = rc;
  cfg->initial.localSize = cfg->output.localSize = ln;
  cfg->initial.localStart = cfg->output.localStart = ls;
  cfg->initial.hasLocalElements = cfg->output.hasLocalElements = ln > 0;
  cfg->allocElements = as;
  cfg->isActive = 1;
  cfg->activeRank = 0;
  cfg->activeSize = 1;
  if (cfg->activeComm != MPI_COMM_NULL) MPI_Comm_free(&cfg->activeComm);
  MPI_Comm_dup(cfg->worldComm, &cfg->activeComm);
  cfg->nodeId = 0;
  cfg->nodeCount = 1;
  free(cfg->hostname);
  free(cfg->deviceName);
  hostAndDevice(&cfg->hostname, &cfg->hostnameLen, &cfg->deviceName, &cfg->deviceNameLen);
  cfg->flags = SHAFFT_CONFIG_RESOLVED;
  cfg->status = 0;
  return ok();
}

int shafft1DInitFromConfig(void* planPtr, shafft_1d_config_t* cfg) {
  if (!planPtr || !cfg) return fail(SHAFFT_ERR_NULLPTR);
  if (!(cfg->flags & SHAFFT_CONFIG_RESOLVED)) {
    int rc = shafftConfig1DResolve(cfg);
    if (rc) return rc;
  }
  return shafft1DInit(planPtr, cfg->globalSize, cfg->initial.localSize, cfg->initial.localStart,
                      cfg->precision, cfg->worldComm);
}

int shafftGetCommunicator(void* planPtr, MPI_Comm* outComm) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  return asPlan(planPtr)->communicator(outComm);
}

// ---- decomposition ---------------------------------------------------------

int shafftConfigurationND(int ndim, int* size, shafft_t precision, int* commDims, int* nda,
                          size_t* subsize, size_t* offset, int* commSize,
                          shafft_decomposition_strategy_t, size_t memLimit, MPI_Comm cComm) {
  if (!size || !commDims || !nda || !subsize || !offset || !commSize) return fail(SHAFFT_ERR_NULLPTR);
  if (ndim < 1) return fail(SHAFFT_ERR_INVALID_DIM);
  if (precision != SHAFFT_C2C && precision != SHAFFT_Z2Z) return fail(SHAFFT_ERR_INVALID_FFTTYPE);
  int world = 0;
  int rc = MPI_Comm_size(cComm, &world);
  if (rc != MPI_SUCCESS) return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
  for (int i = 0; i < ndim; ++i)
    if (size[i] < 1) return fail(SHAFFT_ERR_INVALID_DIM);
  // With one rank every fallback of the reference's cascade
  // (src/cpp/configuration.cpp:530-600) resolves to the trivial grid.
  const size_t esz = (precision == SHAFFT_Z2Z) ? 16 : 8;
  if (memLimit) {
    unsigned __int128 bytes = 2 * (unsigned __int128)esz;  // data + work buffers
    for (int i = 0; i < ndim; ++i) bytes *= (unsigned __int128)size[i];
    if (bytes > (unsigned __int128)memLimit)
      return fail(SHAFFT_ERR_INVALID_DECOMP, SHAFFT_ERRSRC_NONE, 0,
                  "tensor needs more than memLimit=%zu bytes on the single rank", memLimit);
  }
  for (int i = 0; i < ndim; ++i) {
    commDims[i] = 1;
    subsize[i] = (size_t)size[i];
    offset[i] = 0;
  }
  *nda = 0;
  *commSize = world >= 1 ? 1 : 0;
  return ok();
}

int shafftNDCreate(void** outPlan) {
  if (!outPlan) return fail(SHAFFT_ERR_NULLPTR);
  *outPlan = nullptr;
  auto* p = new (std::nothrow) FFTNDPlan();
  if (!p) return fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_SYSTEM);
  *outPlan = static_cast<PlanBase*>(p);
  return ok();
}

int shafftNDInit(void* planPtr, int ndim, int commDims[], int dimensions[], shafft_t precision,
                 MPI_Comm cComm, shafft_transform_layout_t output_policy) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  PlanBase* b = asPlan(planPtr);
  if (b->type != shafft::PlanType::PLAN_ND) return fail(SHAFFT_ERR_INVALID_STATE);
  if (precision != SHAFFT_C2C && precision != SHAFFT_Z2Z) return fail(SHAFFT_ERR_INVALID_FFTTYPE);
  // an output policy outside the enum is refused before anything is
  // configured (src/c/shafftc.cpp:42-56, 91-94)
  if (output_policy != SHAFFT_LAYOUT_REDISTRIBUTED && output_policy != SHAFFT_LAYOUT_INITIAL)
    return fail(SHAFFT_ERR_INVALID_LAYOUT);
  return static_cast<FFTNDPlan*>(b)->configure(
      ndim, commDims, dimensions, precision == SHAFFT_Z2Z ? shafft::FFTType::Z2Z : shafft::FFTType::C2C,
      cComm,
      output_policy == SHAFFT_LAYOUT_INITIAL ? shafft::TransformLayout::INITIAL
                                             : shafft::TransformLayout::REDISTRIBUTED);
}

int shafftPlan(void* planPtr) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  PlanBase* b = asPlan(planPtr);
  if (!b->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return b->plan();
}

int shafftDestroy(void** planPtr) {
  if (!planPtr || !*planPtr) return fail(SHAFFT_ERR_NULLPTR);
  delete asPlan(*planPtr);
  *planPtr = nullptr;
  return ok();
}

int shafftGetLayout(void* planPtr, size_t* subsize, size_t* offset, shafft_tensor_layout_t) {
  if (!planPtr || !asPlan(planPtr)->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  if (!subsize || !offset) return fail(SHAFFT_ERR_NULLPTR);
  return fillLayout(asPlan(planPtr), subsize, offset);
}

int shafftGetAxes(void* planPtr, int* ca, int* da, shafft_tensor_layout_t) {
  if (!planPtr || !asPlan(planPtr)->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  return fillAxes(asPlan(planPtr), ca, da);
}

int shafftGetAllocSize(void* plan, size_t* localAllocSize) {
  if (!localAllocSize) return fail(SHAFFT_ERR_NULLPTR);
  if (!plan || !asPlan(plan)->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  *localAllocSize = asPlan(plan)->allocSize();
  return ok();
}

int shafftGetGlobalSize(void* plan, size_t* globalSize) {
  if (!globalSize) return fail(SHAFFT_ERR_NULLPTR);
  if (!plan || !asPlan(plan)->configured) return fail(SHAFFT_ERR_PLAN_NOT_INIT);
  *globalSize = asPlan(plan)->globalSize();
  return ok();
}

int shafftIsConfigured(void* plan, int* configured) {
  if (!configured) return fail(SHAFFT_ERR_NULLPTR);
  *configured = (plan && asPlan(plan)->configured) ? 1 : 0;
  return ok();
}

int shafftIsActive(void* plan, int* active) {
  if (!active) return fail(SHAFFT_ERR_NULLPTR);
  *active = (plan && asPlan(plan)->configured && asPlan(plan)->active) ? 1 : 0;
  return ok();
}

int shafftSetBuffers(void* planPtr, void* data, void* work) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  return asPlan(planPtr)->setBuffers(data, work);
}

int shafftGetBuffers(void* planPtr, void** data, void** work) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  return asPlan(planPtr)->getBuffers(data, work);
}

int shafftExecute(void* planPtr, shafft_direction_t direction) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  if (direction != SHAFFT_FORWARD && direction != SHAFFT_BACKWARD) return fail(SHAFFT_ERR_INVALID_DIM);
  return asPlan(planPtr)->execute(
      direction == SHAFFT_FORWARD ? shafft::FFTDirection::FORWARD : shafft::FFTDirection::BACKWARD, false);
}

int shafftExecuteNormalized(void* planPtr, shafft_direction_t direction) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  if (direction != SHAFFT_FORWARD && direction != SHAFFT_BACKWARD) return fail(SHAFFT_ERR_INVALID_DIM);
  return asPlan(planPtr)->execute(
      direction == SHAFFT_FORWARD ? shafft::FFTDirection::FORWARD : shafft::FFTDirection::BACKWARD, true);
}

int shafftNormalize(void* planPtr) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  return asPlan(planPtr)->normalize();
}

int shafftConfiguration1D(size_t N, size_t* localN, size_t* localStart, size_t* localAllocSize,
                          shafft_t precision, MPI_Comm cComm) {
  if (!localN || !localStart || !localAllocSize) return fail(SHAFFT_ERR_NULLPTR);
  (void)precision;
  int world = 0;
  int rc = MPI_Comm_size(cComm, &world);
  if (rc != MPI_SUCCESS) return fail(SHAFFT_ERR_MPI, SHAFFT_ERRSRC_MPI, rc);
  // one rank: the whole sequence, no padding (reference
  // src/cpp/fft/hipfft_method/fft1d_method.hip:331-414 with P = 1)
  *localN = N;
  *localStart = 0;
  *localAllocSize = N;
  return ok();
}

int shafft1DCreate(void** outPlan) {
  if (!outPlan) return fail(SHAFFT_ERR_NULLPTR);
  *outPlan = nullptr;
  auto* p = new (std::nothrow) FFT1DPlan();
  if (!p) return fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_SYSTEM);
  *outPlan = static_cast<PlanBase*>(p);
  return ok();
}

int shafft1DInit(void* planPtr, size_t N, size_t, size_t, shafft_t precision, MPI_Comm cComm) {
  if (!planPtr) return fail(SHAFFT_ERR_NULLPTR);
  PlanBase* b = asPlan(planPtr);
  if (b->type != shafft::PlanType::PLAN_1D) return fail(SHAFFT_ERR_INVALID_STATE);
  if (precision != SHAFFT_C2C && precision != SHAFFT_Z2Z) return fail(SHAFFT_ERR_INVALID_FFTTYPE);
  return static_cast<FFT1DPlan*>(b)->configure(
      N, precision == SHAFFT_Z2Z ? shafft::FFTType::Z2Z : shafft::FFTType::C2C, cComm);
}

// ---- buffers ---------------------------------------------------------------

static int allocBytes(size_t count, size_t esz, void** buf) {
  if (!buf) return fail(SHAFFT_ERR_NULLPTR);
  *buf = nullptr;
  if (count == 0) return ok();
  if (count > SIZE_MAX / esz) return fail(SHAFFT_ERR_SIZE_OVERFLOW);
  int rc = shafft_sm100_malloc(buf, count * esz);
  if (rc) {
    *buf = nullptr;
    return fail(SHAFFT_ERR_ALLOC, SHAFFT_ERRSRC_HIP, shafft_sm100_last_cuda_error(), "%s",
                shafft_sm100_last_error_message());
  }
  return ok();
}
static int freeBytes(void* buf) {
  if (!buf) return ok();
  int rc = shafft_sm100_free(buf);
  if (rc) return backend_fail(rc, "free");
  return ok();
}
static int copyBytes(void* dst, const void* src, size_t bytes, int kind) {
  if (!bytes) return ok();
  if (!dst || !src) return fail(SHAFFT_ERR_NULLPTR);
  int rc = shafft_sm100_memcpy(dst, src, bytes, kind, nullptr);
  if (rc) return backend_fail(rc, "copy");
  return ok();
}

int shafftAllocBufferF(size_t count, void** buf) { return allocBytes(count, 8, buf); }
int shafftAllocBufferD(size_t count, void** buf) { return allocBytes(count, 16, buf); }
int shafftFreeBufferF(void* buf) { return freeBytes(buf); }
int shafftFreeBufferD(void* buf) { return freeBytes(buf); }
int shafftCopyToBufferF(void* dst, const void* src, size_t count) {
  return copyBytes(dst, src, count * 8, SHAFFT_SM100_H2D);
}
int shafftCopyToBufferD(void* dst, const void* src, size_t count) {
  return copyBytes(dst, src, count * 16, SHAFFT_SM100_H2D);
}
int shafftCopyFromBufferF(void* dst, const void* src, size_t count) {
  return copyBytes(dst, src, count * 8, SHAFFT_SM100_D2H);
}
int shafftCopyFromBufferD(void* dst, const void* src, size_t count) {
  return copyBytes(dst, src, count * 16, SHAFFT_SM100_D2H);
}

const char* shafftGetBackendName(void) { return SHAFFT_BACKEND_NAME; }

void shafftGetVersion(int* major, int* minor, int* patch) {
  if (major) *major = SHAFFT_VERSION_MAJOR;
  if (minor) *minor = SHAFFT_VERSION_MINOR;
  if (patch) *patch = SHAFFT_VERSION_PATCH;
}

const char* shafftGetVersionString(void) {
  return SHAFFT_STRINGIFY(SHAFFT_VERSION_MAJOR) "." SHAFFT_STRINGIFY(
      SHAFFT_VERSION_MINOR) "." SHAFFT_STRINGIFY(SHAFFT_VERSION_PATCH) SHAFFT_VERSION_SUFFIX;
}

int shafftFinalize(void) { return ok(); }

}  // extern "C"
