// C++ caller of the SHAFFT API (include/shafft/shafft.hpp), host-side
// behaviour only: init/plan state errors, move semantics, release
// idempotence, FFT1D argument checks and the decomposition queries
// (reference semantics: src/cpp/shafft.cpp:18-62, 174-175, 918-945;
// src/cpp/shafft_internal.cpp:37-60; tests/unit/test_errors.cpp:166-192).
// Prints one line per check and "<n> failure(s)" at the end; exit status is
// the failure count.
#include <shafft/shafft.hpp>

#include <climits>
#include <cstdio>
#include <utility>
#include <vector>

namespace {
int failures = 0;

void check(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "PASS" : "FAIL", what);
  if (!ok) ++failures;
}

int st(shafft::Status s) { return static_cast<int>(s); }
}  // namespace

int main() {
  using shafft::FFT1D;
  using shafft::FFTND;
  using shafft::FFTType;
  using shafft::Status;

  check(std::string(shafft::getBackendName()) == "sm100", "backend name");
  check(std::string(shafft::getVersionString()) == "1.1.0-alpha", "version string");

  {  // state machine before and after init
    FFTND p;
    check(!p.isConfigured() && !p, "fresh plan is not configured");
    check(p.plan() == st(Status::ERR_PLAN_NOT_INIT), "plan before init");
    check(p.execute(shafft::FFTDirection::FORWARD) == st(Status::ERR_PLAN_NOT_INIT), "execute before plan");
    check(p.normalize() == st(Status::ERR_PLAN_NOT_INIT), "normalize before plan");
    check(p.init({1, 1, 1}, {64, 64, 32}, FFTType::C2C, MPI_COMM_WORLD) == 0, "init 64x64x32");
    check(p.isConfigured() && p.allocSize() == 64 * 64 * 32, "configured, allocSize = N");
    check(p.init({1, 1, 1}, {64, 64, 32}, FFTType::C2C, MPI_COMM_WORLD) == st(Status::ERR_INVALID_STATE),
          "re-init is an invalid state");
    check(p.execute(shafft::FFTDirection::FORWARD) == st(Status::ERR_PLAN_NOT_INIT),
          "execute after init, before plan");
    MPI_Comm c = MPI_COMM_NULL;
    check(p.getCommunicator(&c) == 0 && c != MPI_COMM_NULL, "communicator available after init");
    // an active rank must hand over both buffers (src/cpp/shafft_internal.cpp:505-523)
    check(p.setBuffersRaw(nullptr, nullptr) == st(Status::ERR_NULLPTR), "null buffers on an active rank");
    void* d = nullptr;
    void* w = nullptr;
    check(p.getBuffersRaw(&d, &w) == st(Status::ERR_NO_BUFFER) && !d && !w,
          "getBuffers on an active rank without buffers");

    // move construction and assignment leave the source uninitialised
    FFTND q(std::move(p));
    check(q.isConfigured() && q.allocSize() == 64 * 64 * 32, "moved-to plan keeps the configuration");
    check(!p.isConfigured() && p.state() == shafft::PlanState::UNINITIALIZED, "moved-from plan is uninitialised");
    check(p.plan() == st(Status::ERR_PLAN_NOT_INIT), "moved-from plan cannot plan");
    FFTND r;
    r = std::move(q);
    check(r.isConfigured() && !q.isConfigured(), "move assignment");
    r.release();
    check(!r.isConfigured(), "release returns to uninitialised");
    r.release();  // idempotent
    check(!r.isConfigured(), "double release is safe");
    check(r.init({1, 1}, {16, 16}, FFTType::Z2Z, MPI_COMM_WORLD) == 0, "init again after release");
  }

  {  // an inactive rank (MPI_COMM_NULL) owns nothing and may pass null buffers
    FFTND p;
    check(p.init({1, 1}, {8, 8}, FFTType::C2C, MPI_COMM_NULL) == 0 && !p.isActive() && p.allocSize() == 0,
          "inactive rank");
    check(p.setBuffersRaw(nullptr, nullptr) == 0, "inactive rank accepts null buffers");
  }

  {  // FFTND argument errors
    FFTND p;
    check(p.init({1, 1}, {8, 8, 8}, FFTType::C2C, MPI_COMM_WORLD) == st(Status::ERR_DIM_MISMATCH),
          "commDims / dims size mismatch");
    FFTND q;
    check(q.init({1, 1}, {(size_t)INT_MAX + 1, 4}, FFTType::C2C, MPI_COMM_WORLD) ==
              st(Status::ERR_SIZE_OVERFLOW),
          "dimension above INT_MAX");
    FFTND s;
    check(s.init({2, 1}, {8, 8}, FFTType::C2C, MPI_COMM_WORLD) == st(Status::ERR_INVALID_DECOMP),
          "grid of 2 ranks on a 1-rank communicator");
  }

  {  // FFT1D
    FFT1D p;
    check(p.init(0, 0, 0, FFTType::C2C, MPI_COMM_WORLD) == st(Status::ERR_INVALID_DIM), "FFT1D of length 0");
    FFT1D q;
    check(q.init(4096, 4096, 0, FFTType::Z2Z, MPI_COMM_WORLD) == 0 && q.allocSize() == 4096, "FFT1D init");
    FFT1D r(std::move(q));
    check(r.allocSize() == 4096 && !q.isConfigured(), "FFT1D move leaves the source uninitialised");
    r.release();
    r.release();
    check(!r.isConfigured(), "FFT1D double release is safe");
  }

  {  // decomposition queries on one rank
    std::vector<int> cd(3, 0);
    std::vector<size_t> sub, off;
    int nda = -1, cs = 0;
    // output vectors must come sized to ndim (src/cpp/shafft.cpp:374-377)
    check(shafft::configurationND({64, 64, 32}, FFTType::C2C, cd, nda, sub, off, cs,
                                  shafft::DecompositionStrategy::MAXIMIZE_NDA, 0, MPI_COMM_WORLD) ==
              st(Status::ERR_DIM_MISMATCH),
          "configurationND with unsized output vectors");
    sub.assign(3, 0);
    off.assign(3, 0);
    const int rc = shafft::configurationND({64, 64, 32}, FFTType::C2C, cd, nda, sub, off, cs,
                                           shafft::DecompositionStrategy::MAXIMIZE_NDA, 0, MPI_COMM_WORLD);
    check(rc == 0 && cd == std::vector<int>({1, 1, 1}) && nda == 0 && cs == 1 &&
              sub == std::vector<size_t>({64, 64, 32}),
          "configurationND on one rank");
    size_t ln = 0, ls = 1;
    check(shafft::configuration1D(1000003, ln, ls, FFTType::C2C, MPI_COMM_WORLD) == 0 && ln == 1000003 &&
              ls == 0,
          "configuration1D on one rank");
  }

  std::printf("%d failure(s)\n", failures);
  return failures;
}
