// abi.cpp -- the C ABI of libket_b200.so (declared in include/ket_b200.h).
//
// Every entry point converts exceptions into KETGPU_ERR_* codes with a
// thread-local message, validates its arguments on the host before any
// launch, and leaves the caller's current CUDA device unchanged.
#include <cuda_runtime.h>

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <barrier>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

#define KB_API extern "C" __attribute__((visibility("default")))

namespace kb {

std::atomic<uint64_t> g_launches{0};

namespace {
thread_local std::string t_err;
}

void fail(int code, const std::string& msg) { throw Error(code, msg); }
void set_last_error(const char* msg) { t_err = msg; }

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const int code = (e == cudaErrorMemoryAllocation) ? KETGPU_ERR_OOM : KETGPU_ERR_CUDA;
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceGuard::DeviceGuard(int dev) {
  KB_CUDA(cudaGetDevice(&prev));
  if (prev != dev) KB_CUDA(cudaSetDevice(dev));
}
DeviceGuard::~DeviceGuard() {
  int cur = -1;
  if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
}

Plan::~Plan() {
  if (device >= 0) {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (d_mat64) cudaFree(d_mat64);
    if (d_mat32) cudaFree(d_mat32);
    if (d_tc) cudaFree(d_tc);
    if (d_norm) cudaFree(d_norm);
    if (d_diag) cudaFree(d_diag);
    if (d_runs) cudaFree(d_runs);
    if (prev >= 0) cudaSetDevice(prev);
  }
}

void pauli_masks(int n, const char* pauli, uint64_t& flip, uint64_t& sign, int& q) {
  if (!pauli) fail(KETGPU_ERR_INVALID, "expval: null Pauli string");
  const size_t len = std::strlen(pauli);
  if (len != (size_t)n)
    fail(KETGPU_ERR_INVALID, "expval: Pauli string length must equal the number of qubits");
  flip = 0;
  sign = 0;
  int num_y = 0;
  for (int i = 0; i < n; ++i) {
    char p = pauli[n - 1 - i];  // rightmost character acts on qubit 0
    if (p >= 'a' && p <= 'z') p = (char)(p - ('a' - 'A'));
    const uint64_t bit = uint64_t{1} << i;
    switch (p) {
      case 'I': break;
      case 'X': flip |= bit; break;
      case 'Y': flip |= bit; sign |= bit; ++num_y; break;
      case 'Z': sign |= bit; break;
      default: fail(KETGPU_ERR_INVALID, std::string("expval: invalid Pauli character '") + p + "'");
    }
  }
  q = num_y % 4;
}

void upload_plan_copies(Plan& plan, int device);

// Device copies of a plan's tables, once per plan and device.  They go up
// with cudaMemcpy from pageable host vectors, which may return before the
// data lands; the kernels that read them run on the states' non-blocking
// streams, which do not wait for the legacy stream the copies use, so the
// copies are waited for here.
void upload_plan_matrices(Plan& plan, int device) {
  if (plan.device == device) return;
  upload_plan_copies(plan, device);
  KB_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
}

void upload_plan_copies(Plan& plan, int device) {
  if (plan.device >= 0) fail(KETGPU_ERR_INVALID, "plan was prepared for another device");
  plan.device = device;
  for (const Pass& p : plan.passes)
    if (p.kind == PassKind::NormCapture && !plan.d_norm)
      KB_CUDA(cudaMalloc(&plan.d_norm, sizeof(double) * (2 + kNormBlocks)));
  if (!plan.diags.empty()) {
    std::vector<unsigned char> all, one;
    plan.offdiag.assign(plan.diags.size(), 0);
    for (size_t i = 0; i < plan.diags.size(); ++i) {
      diag_device_data(plan.diags[i], plan.n, plan.precision, one);
      plan.offdiag[i] = all.size();
      all.insert(all.end(), one.begin(), one.end());
      while (all.size() % 256) all.push_back(0);
    }
    KB_CUDA(cudaMalloc(&plan.d_diag, all.size()));
    KB_CUDA(cudaMemcpy(plan.d_diag, all.data(), all.size(), cudaMemcpyHostToDevice));
  }
  if (!plan.runs.empty()) {
    std::vector<unsigned char> all, one;
    plan.offrun.assign(plan.runs.size(), 0);
    for (size_t i = 0; i < plan.runs.size(); ++i) {
      run_device_data(plan.runs[i], plan.precision, one);
      plan.offrun[i] = all.size();
      all.insert(all.end(), one.begin(), one.end());
      while (all.size() % 256) all.push_back(0);
    }
    KB_CUDA(cudaMalloc(&plan.d_runs, all.size()));
    KB_CUDA(cudaMemcpy(plan.d_runs, all.data(), all.size(), cudaMemcpyHostToDevice));
  }
  if (plan.matrices.empty()) return;
  std::vector<double> h64;
  std::vector<float> h32;
  std::vector<uint32_t> htc;
  std::vector<size_t> tc_jobs;
  size_t tc_words = 0;
  plan.off64.assign(plan.matrices.size(), 0);
  plan.off32.assign(plan.matrices.size(), 0);
  plan.offtc.assign(plan.matrices.size(), 0);
  // matrix index -> whether its pass is on the tensor cores
  std::vector<int> kof(plan.matrices.size(), 0);
  std::vector<char> tensor(plan.matrices.size(), 0);
  for (const Pass& p : plan.passes)
    if (p.kind == PassKind::Fused) {
      kof[p.mat_index] = p.k;
      tensor[p.mat_index] = p.tensor;
    }
  for (size_t i = 0; i < plan.matrices.size(); ++i) {
    const std::vector<cplx>& m = plan.matrices[i];
    const int dim = 1 << kof[i];
    if (plan.precision == KETGPU_C128) {
      plan.off64[i] = h64.size() * sizeof(double);
      for (int c = 0; c < dim; ++c)
        for (int r = 0; r < dim; ++r) {
          h64.push_back(m[(size_t)r * dim + c].real());
          h64.push_back(m[(size_t)r * dim + c].imag());
        }
      while (h64.size() % 2) h64.push_back(0);
    } else if (tensor[i]) {
      // place now, build below on host threads
      plan.offtc[i] = tc_words * sizeof(uint32_t);
      tc_jobs.push_back(i);
      tc_words += (tc_image_bytes(kof[i]) / 4 + 63) / 64 * 64;  // 256-byte alignment
    } else {
      plan.off32[i] = h32.size() * sizeof(float);
      for (int c = 0; c < dim; ++c)
        for (int r = 0; r < dim; ++r) {
          h32.push_back((float)m[(size_t)r * dim + c].real());
          h32.push_back((float)m[(size_t)r * dim + c].imag());
        }
      while (h32.size() % 4) h32.push_back(0);
    }
  }
  if (!h64.empty()) {
    KB_CUDA(cudaMalloc(&plan.d_mat64, h64.size() * sizeof(double)));
    KB_CUDA(cudaMemcpy(plan.d_mat64, h64.data(), h64.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (!h32.empty()) {
    KB_CUDA(cudaMalloc(&plan.d_mat32, h32.size() * sizeof(float)));
    KB_CUDA(cudaMemcpy(plan.d_mat32, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (!tc_jobs.empty()) {
    // tensor-core B images (fp16 splits of every entry) on host threads,
    // each written at its place in htc
    htc.assign(tc_words, 0u);
    auto build = [&](size_t i) {
      std::vector<uint32_t> img;
      build_tc_image(plan.matrices[i], kof[i], img);
      std::memcpy(htc.data() + plan.offtc[i] / sizeof(uint32_t), img.data(), img.size() * sizeof(uint32_t));
    };
    const unsigned nt = tc_jobs.size() < 4 ? 1u
                        : std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (nt <= 1) {
      for (size_t i : tc_jobs) build(i);
    } else {
      std::atomic<size_t> next{0};
      std::exception_ptr err;
      std::atomic<bool> failed{false};
      std::vector<std::thread> th;
      for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&] {
          for (size_t j; (j = next.fetch_add(1)) < tc_jobs.size();) {
            try {
              build(tc_jobs[j]);
            } catch (...) {
              if (!failed.exchange(true)) err = std::current_exception();
            }
          }
        });
      for (auto& x : th) x.join();
      if (err) std::rethrow_exception(err);
    }
  }
  if (!htc.empty()) {
    KB_CUDA(cudaMalloc(&plan.d_tc, htc.size() * sizeof(uint32_t)));
    KB_CUDA(cudaMemcpy(plan.d_tc, htc.data(), htc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  }
}

int tc_error_flag(bool reset);

namespace {

State* as_state(ketgpu_state* s) { return reinterpret_cast<State*>(s); }
const State* as_state(const ketgpu_state* s) { return reinterpret_cast<const State*>(s); }
Plan* as_plan(ketgpu_plan* p) { return reinterpret_cast<Plan*>(p); }
const Plan* as_plan(const ketgpu_plan* p) { return reinterpret_cast<const Plan*>(p); }

template <class F>
int guard(F&& f) {
  try {
    f();
    return KETGPU_OK;
  } catch (const Error& e) {
    t_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    t_err = "host allocation failed";
    return KETGPU_ERR_OOM;
  } catch (const std::exception& e) {
    t_err = e.what();
    return KETGPU_ERR_LOGIC;
  }
}

void need(bool cond, const char* msg) {
  if (!cond) fail(KETGPU_ERR_INVALID, msg);
}

// Parallel host conversion helpers for the host<->device complex128 copies.
template <class F>
void parallel_chunks(uint64_t count, F&& f) {
  unsigned nt = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (count < (1u << 20)) nt = 1;
  std::vector<std::thread> th;
  const uint64_t per = (count + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const uint64_t lo = t * per, hi = std::min(count, lo + per);
    if (lo >= hi) break;
    th.emplace_back([&, lo, hi] { f(lo, hi); });
  }
  for (auto& x : th) x.join();
}

struct Pinned {
  void* p = nullptr;
  explicit Pinned(size_t b) { KB_CUDA(cudaMallocHost(&p, b)); }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

constexpr uint64_t kChunk = uint64_t{1} << 24;  // amplitudes per staged upload copy

// complex64 -> complex128 widening of n floats (re, im interleaved).  The
// AVX-512 form widens 8 floats per instruction and writes with non-temporal
// stores (no read-for-ownership of the destination lines), which matters
// because the destination is twice the size of everything else that moves.
__attribute__((target("avx512f"))) void widen_avx512(const float* src, double* dst, uint64_t n) {
  uint64_t i = 0;
  while (i < n && (reinterpret_cast<uintptr_t>(dst + i) & 63)) {
    dst[i] = (double)src[i];
    ++i;
  }
  for (; i + 8 <= n; i += 8) _mm512_stream_pd(dst + i, _mm512_cvtps_pd(_mm256_loadu_ps(src + i)));
  for (; i < n; ++i) dst[i] = (double)src[i];
  _mm_sfence();
}

void widen_scalar(const float* src, double* dst, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) dst[i] = (double)src[i];
}

bool have_avx512() {
  static const bool v = __builtin_cpu_supports("avx512f");
  return v;
}

// Pinned staging for complex64 downloads, kept for the life of the process:
// a ring of down_ring() buffers of down_chunk() amplitudes (default 4 x 16 MB),
// all but one of them in flight.  One download at a time uses it.  At 30
// qubits 4 x 16 MB matched the raw copy (157-160 ms against 162 ms to pinned
// memory); 3 x 32 MB took 181-188 ms and 4 x 8 MB 213-243 ms, the widening
// no longer hidden behind the copy.  KETGPU_DOWN_CHUNK_MB and
// KETGPU_DOWN_RING override the shape (read once).
uint64_t env_u64(const char* name, uint64_t def, uint64_t lo, uint64_t hi) {
  const char* e = std::getenv(name);
  if (!e) return def;
  const uint64_t v = std::strtoull(e, nullptr, 10);
  return v < lo ? lo : (v > hi ? hi : v);
}
uint64_t down_chunk() {
  static const uint64_t v = env_u64("KETGPU_DOWN_CHUNK_MB", 16, 1, 256) * (uint64_t{1} << 20) / 8;
  return v;
}
int down_ring() {
  static const int v = (int)env_u64("KETGPU_DOWN_RING", 4, 2, 16);
  return v;
}
std::mutex g_stage_mu;
void* g_stage = nullptr;

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Where a complex64 download spends the calling thread's time: waiting for
// device-to-host copies, and widening its share of each chunk.
struct DownloadTimes {
  double copy_wait_ms = 0.0, widen_ms = 0.0;
};

// Phase times of the calling thread's last ketgpu_run (ketgpu_run_last_profile).
thread_local double t_run_profile[6] = {0, 0, 0, 0, 0, 0};

void download(const State& s, uint64_t first, uint64_t count, double* out, DownloadTimes* times = nullptr) {
  if (s.precision == KETGPU_C128) {
    KB_CUDA(cudaMemcpyAsync(out, static_cast<const double2*>(s.amps) + first, count * 16,
                            cudaMemcpyDeviceToHost, s.stream));
    KB_CUDA(cudaStreamSynchronize(s.stream));
    return;
  }
  std::lock_guard<std::mutex> lock(g_stage_mu);
  const uint64_t chunk = down_chunk();
  const int ring = down_ring();
  if (!g_stage) KB_CUDA(cudaMallocHost(&g_stage, ring * chunk * 8));
  std::vector<float2*> buf(ring);
  for (int b = 0; b < ring; ++b) buf[b] = static_cast<float2*>(g_stage) + b * chunk;
  std::vector<cudaEvent_t> ev(ring);
  for (auto& e : ev) KB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  const uint64_t nchunks = (count + chunk - 1) / chunk;
  cudaError_t err = cudaSuccess;  // no throw while the workers run
  auto issue = [&](uint64_t c) {
    const uint64_t lo = c * chunk, len = std::min(chunk, count - lo);
    cudaError_t e = cudaMemcpyAsync(buf[c % ring], static_cast<const float2*>(s.amps) + first + lo, len * 8,
                                    cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[c % ring], s.stream);
    if (e != cudaSuccess && err == cudaSuccess) err = e;
  };
  // Chunk c is widened by every worker while chunks c+1 .. c+ring-1 are in
  // flight.  The workers start once per download and step through the
  // chunks between two barriers; the calling thread is worker 0 and also
  // issues the copies.
  const unsigned nt = count < (uint64_t{1} << 20) ? 1u
                                                  : std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  const bool wide = have_avx512();
  auto slice = [&](unsigned t, uint64_t c) {
    const uint64_t lo = c * chunk, len = std::min(chunk, count - lo);
    // in floats, rounded to 16 floats (64 bytes of output) per worker
    const uint64_t nf = 2 * len, per = ((nf + nt - 1) / nt + 15) / 16 * 16;
    const uint64_t a = std::min(nf, t * per), b = std::min(nf, a + per);
    if (b > a)
      (wide ? widen_avx512 : widen_scalar)(reinterpret_cast<const float*>(buf[c % ring]) + a, out + 2 * lo + a, b - a);
  };
  std::barrier sync(nt);
  auto work = [&](unsigned t) {
    for (uint64_t c = 0; c < nchunks; ++c) {
      sync.arrive_and_wait();  // chunk c has landed
      slice(t, c);
      sync.arrive_and_wait();  // chunk c is consumed
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
  for (uint64_t c = 0; c < std::min<uint64_t>(ring - 1, nchunks); ++c) issue(c);
  for (uint64_t c = 0; c < nchunks; ++c) {
    const auto w0 = std::chrono::steady_clock::now();
    if (err == cudaSuccess) {
      const cudaError_t e = cudaEventSynchronize(ev[c % ring]);
      if (e != cudaSuccess) err = e;
    }
    if (times) times->copy_wait_ms += ms_since(w0);
    if (c + ring - 1 < nchunks && err == cudaSuccess) issue(c + ring - 1);
    sync.arrive_and_wait();
    const auto s0 = std::chrono::steady_clock::now();
    slice(0, c);
    if (times) times->widen_ms += ms_since(s0);
    sync.arrive_and_wait();
  }
  for (auto& x : th) x.join();
  for (auto& e : ev) cudaEventDestroy(e);
  check_cuda(err, "download");
}

void upload(State& s, uint64_t first, uint64_t count, const double* in) {
  s.touch();
  if (s.precision == KETGPU_C128) {
    KB_CUDA(cudaMemcpyAsync(static_cast<double2*>(s.amps) + first, in, count * 16, cudaMemcpyHostToDevice,
                            s.stream));
    KB_CUDA(cudaStreamSynchronize(s.stream));
    return;
  }
  const uint64_t chunk = std::min<uint64_t>(kChunk, std::max<uint64_t>(count, 1));
  Pinned stage(chunk * 8);
  float2* buf = static_cast<float2*>(stage.p);
  for (uint64_t lo = 0; lo < count; lo += chunk) {
    const uint64_t len = std::min(chunk, count - lo);
    parallel_chunks(len, [&](uint64_t a, uint64_t b) {
      for (uint64_t i = a; i < b; ++i) buf[i] = make_float2((float)in[2 * (lo + i)], (float)in[2 * (lo + i) + 1]);
    });
    KB_CUDA(cudaMemcpyAsync(static_cast<float2*>(s.amps) + first + lo, buf, len * 8, cudaMemcpyHostToDevice,
                            s.stream));
    KB_CUDA(cudaStreamSynchronize(s.stream));
  }
}

void execute(const Plan& plan, State& s) {
  need(plan.n == s.n, "plan and state have different qubit counts");
  need(plan.precision == s.precision, "plan and state have different precisions");
  upload_plan_matrices(const_cast<Plan&>(plan), s.device);
  for (const Pass& p : plan.passes) launch_pass(s, plan, p);
}

void check_tc_flag() {
  if (tc_error_flag(true))
    fail(KETGPU_ERR_TIMEOUT, "tensor-core block kernel timed out waiting on its MMA barrier");
}

}  // namespace

// Create a state on the current device (used by adjoint.cu too).
// The device state of the last ketgpu_run call, kept for the next call of
// the same size and device.  Freeing a 30-qubit state (8 GiB) costs
// 150-700 ms in cudaFree, more than downloading it.  Guarded by g_run_mu;
// a call takes the state out while it runs.
std::mutex g_run_mu;
State* g_run_state = nullptr;

void destroy_state(State* s);

void release_run_state() {
  State* s = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_run_mu);
    std::swap(s, g_run_state);
  }
  destroy_state(s);
}

State* create_state(int n, int precision) {
  if (n < 0 || n > 40) fail(KETGPU_ERR_INVALID, "n_qubits must be in [0, 40]");
  if (precision != KETGPU_C64 && precision != KETGPU_C128)
    fail(KETGPU_ERR_INVALID, "precision must be KETGPU_C64 or KETGPU_C128");
  auto st = std::make_unique<State>();
  st->n = n;
  st->precision = precision;
  KB_CUDA(cudaGetDevice(&st->device));
  const size_t bytes = (size_t)st->dim() * st->amp_bytes();
  size_t free_b = 0, total_b = 0;
  KB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes > free_b) {  // give back ketgpu_run's kept state first
    release_run_state();
    KB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  }
  if (bytes > free_b)
    fail(KETGPU_ERR_OOM, "state of " + std::to_string(bytes) + " bytes exceeds free device memory (" +
                             std::to_string(free_b) + ")");
  KB_CUDA(cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking));
  const cudaError_t e = cudaMalloc(&st->amps, bytes);
  if (e != cudaSuccess) {
    cudaStreamDestroy(st->stream);
    check_cuda(e, "cudaMalloc(state)");
  }
  std::unique_ptr<State, void (*)(State*)> guard_st(st.release(), destroy_state);
  noalloc_prepare(guard_st->device);
  set_ground(*guard_st);
  return guard_st.release();
}

void destroy_state(State* s) {
  if (!s) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->tree) cudaFree(s->tree);
  if (s->amps) cudaFree(s->amps);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (prev >= 0) cudaSetDevice(prev);
  delete s;
}

void execute_plan(const Plan& plan, State& s) { execute(plan, s); }

}  // namespace kb

using namespace kb;

KB_API const char* ketgpu_last_error(void) { return t_err.c_str(); }
KB_API int ketgpu_abi_version(void) { return KETGPU_ABI_VERSION; }
KB_API uint64_t ketgpu_launch_count(void) { return g_launches.load(); }

KB_API int ketgpu_state_create(int32_t n_qubits, int32_t precision, ketgpu_state** out) {
  return guard([&] {
    need(out != nullptr, "out is null");
    *out = reinterpret_cast<ketgpu_state*>(create_state(n_qubits, precision));
  });
}

KB_API int ketgpu_state_destroy(ketgpu_state* s) {
  return guard([&] { destroy_state(as_state(s)); });
}

KB_API int ketgpu_state_reset(ketgpu_state* s) {
  return guard([&] {
    need(s != nullptr, "state is null");
    DeviceGuard g(as_state(s)->device);
    set_ground(*as_state(s));
    KB_CUDA(cudaStreamSynchronize(as_state(s)->stream));
  });
}

KB_API int ketgpu_state_info(const ketgpu_state* s, int32_t* n, int32_t* precision) {
  return guard([&] {
    need(s != nullptr, "state is null");
    if (n) *n = as_state(s)->n;
    if (precision) *precision = as_state(s)->precision;
  });
}

// Handing out the pointer counts as a write: the caller may change the
// amplitudes through it, so a cached sampling tree is not reused.
KB_API void* ketgpu_state_device_ptr(const ketgpu_state* s) {
  if (!s) return nullptr;
  as_state(s)->touch();
  return as_state(s)->amps;
}

KB_API int ketgpu_state_download(const ketgpu_state* s, uint64_t first, uint64_t count, double* out) {
  return guard([&] {
    need(s != nullptr && (out != nullptr || count == 0), "null argument");
    const State& st = *as_state(s);
    if (first > st.dim() || count > st.dim() - first)
      fail(KETGPU_ERR_OUT_OF_RANGE, "amplitude range outside the state");
    DeviceGuard g(st.device);
    download(st, first, count, out);
  });
}

KB_API int ketgpu_state_download_raw(const ketgpu_state* s, uint64_t first, uint64_t count, void* out) {
  return guard([&] {
    need(s != nullptr && (out != nullptr || count == 0), "null argument");
    const State& st = *as_state(s);
    if (first > st.dim() || count > st.dim() - first)
      fail(KETGPU_ERR_OUT_OF_RANGE, "amplitude range outside the state");
    DeviceGuard g(st.device);
    const size_t b = st.amp_bytes();
    KB_CUDA(cudaMemcpyAsync(out, static_cast<const char*>(st.amps) + first * b, count * b, cudaMemcpyDeviceToHost,
                            st.stream));
    KB_CUDA(cudaStreamSynchronize(st.stream));
  });
}

KB_API int ketgpu_state_upload(ketgpu_state* s, uint64_t first, uint64_t count, const double* in) {
  return guard([&] {
    need(s != nullptr && (in != nullptr || count == 0), "null argument");
    State& st = *as_state(s);
    if (first > st.dim() || count > st.dim() - first)
      fail(KETGPU_ERR_OUT_OF_RANGE, "amplitude range outside the state");
    DeviceGuard g(st.device);
    upload(st, first, count, in);
  });
}

KB_API int ketgpu_state_copy(const ketgpu_state* src, ketgpu_state* dst) {
  return guard([&] {
    need(src && dst, "null state");
    const State& a = *as_state(src);
    State& b = *as_state(dst);
    need(a.n == b.n && a.precision == b.precision, "states differ in size or precision");
    DeviceGuard g(b.device);
    b.touch();
    KB_CUDA(cudaStreamSynchronize(a.stream));
    KB_CUDA(cudaMemcpyAsync(b.amps, a.amps, a.dim() * a.amp_bytes(), cudaMemcpyDefault, b.stream));
    KB_CUDA(cudaStreamSynchronize(b.stream));
  });
}

KB_API int ketgpu_state_synchronize(ketgpu_state* s) {
  return guard([&] {
    need(s != nullptr, "state is null");
    DeviceGuard g(as_state(s)->device);
    KB_CUDA(cudaStreamSynchronize(as_state(s)->stream));
    check_tc_flag();
  });
}

KB_API int ketgpu_plan_create(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const ketgpu_options* opt,
                              ketgpu_plan** out) {
  return guard([&] {
    need(out != nullptr, "out is null");
    need(ops != nullptr || n_ops == 0, "ops is null");
    if (n < 0 || n > 40) fail(KETGPU_ERR_INVALID, "n_qubits must be in [0, 40]");
    validate_ops(n, ops, n_ops);
    auto plan = std::make_unique<Plan>();
    build_plan(*plan, n, ops, n_ops, resolve_options(opt));
    *out = reinterpret_cast<ketgpu_plan*>(plan.release());
  });
}

KB_API int ketgpu_plan_destroy(ketgpu_plan* p) {
  return guard([&] { delete as_plan(p); });
}

KB_API int ketgpu_plan_stats_get(const ketgpu_plan* p, ketgpu_plan_stats* out) {
  return guard([&] {
    need(p && out, "null argument");
    *out = as_plan(p)->stats;
  });
}

KB_API int ketgpu_plan_execute(const ketgpu_plan* p, ketgpu_state* s) {
  return guard([&] {
    need(p && s, "null argument");
    DeviceGuard g(as_state(s)->device);
    execute(*as_plan(p), *as_state(s));
  });
}

KB_API int ketgpu_apply(ketgpu_state* s, const ketgpu_op* ops, uint64_t n_ops, const ketgpu_options* opt) {
  return guard([&] {
    need(s != nullptr, "state is null");
    need(ops != nullptr || n_ops == 0, "ops is null");
    State& st = *as_state(s);
    validate_ops(st.n, ops, n_ops);
    PlanOptions o = resolve_options(opt);
    if (opt == nullptr) o.precision = st.precision;
    need(o.precision == st.precision, "options precision differs from the state's");
    Plan plan;
    build_plan(plan, st.n, ops, n_ops, o);
    DeviceGuard g(st.device);
    execute(plan, st);
    KB_CUDA(cudaStreamSynchronize(st.stream));
    check_tc_flag();
  });
}

KB_API int ketgpu_run(int32_t n, const ketgpu_op* ops, uint64_t n_ops, const ketgpu_options* opt,
                      double* out_c128) {
  return guard([&] {
    need(out_c128 != nullptr, "out is null");
    need(ops != nullptr || n_ops == 0, "ops is null");
    if (n < 0 || n > 40) fail(KETGPU_ERR_INVALID, "n_qubits must be in [0, 40]");
    const auto t0 = std::chrono::steady_clock::now();
    std::fill(t_run_profile, t_run_profile + 6, 0.0);
    validate_ops(n, ops, n_ops);
    const PlanOptions o = resolve_options(opt);
    Plan plan;
    build_plan(plan, n, ops, n_ops, o);
    const double plan_ms = ms_since(t0);
    const auto t1 = std::chrono::steady_clock::now();
    State* kept = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_run_mu);
      std::swap(kept, g_run_state);
    }
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    std::unique_ptr<State, void (*)(State*)> st(nullptr, destroy_state);
    if (kept && kept->n == n && kept->precision == o.precision && kept->device == dev) {
      st.reset(kept);
      set_ground(*st);
    } else {
      destroy_state(kept);
      st.reset(create_state(n, o.precision));
    }
    const double state_ms = ms_since(t1);
    const auto t2 = std::chrono::steady_clock::now();
    execute(plan, *st);
    KB_CUDA(cudaStreamSynchronize(st->stream));
    const double exec_ms = ms_since(t2);
    const auto t3 = std::chrono::steady_clock::now();
    DownloadTimes dt;
    download(*st, 0, st->dim(), out_c128, &dt);
    const double down_ms = ms_since(t3);
    check_tc_flag();
    const double prof[6] = {plan_ms, state_ms, exec_ms, down_ms, dt.copy_wait_ms, dt.widen_ms};
    std::copy(prof, prof + 6, t_run_profile);
    std::lock_guard<std::mutex> lk(g_run_mu);  // keep it for the next call
    if (!g_run_state) g_run_state = st.release();
  });
}

KB_API int ketgpu_run_last_profile(double* out6) {
  return guard([&] {
    need(out6 != nullptr, "out is null");
    std::copy(t_run_profile, t_run_profile + 6, out6);
  });
}

KB_API int ketgpu_release_cache(void) {
  return guard([&] { release_run_state(); });
}

KB_API int ketgpu_norm(const ketgpu_state* s, double* out) {
  return guard([&] {
    need(s && out, "null argument");
    DeviceGuard g(as_state(s)->device);
    *out = reduce_norm(*as_state(s));
  });
}

KB_API int ketgpu_inner(const ketgpu_state* a, const ketgpu_state* b, double* re, double* im) {
  return guard([&] {
    need(a && b, "null state");
    need(as_state(a)->n == as_state(b)->n && as_state(a)->precision == as_state(b)->precision,
         "states differ in size or precision");
    DeviceGuard g(as_state(a)->device);
    const cplx v = reduce_inner(*as_state(a), *as_state(b));
    if (re) *re = v.real();
    if (im) *im = v.imag();
  });
}

KB_API int ketgpu_expval_terms(const ketgpu_state* s, const char* const* paulis, uint64_t n_terms, double* out) {
  return guard([&] {
    need(s != nullptr, "state is null");
    need((paulis && out) || n_terms == 0, "null argument");
    const State& st = *as_state(s);
    std::vector<uint64_t> flip(n_terms), sign(n_terms);
    std::vector<int> q(n_terms);
    for (uint64_t t = 0; t < n_terms; ++t) pauli_masks(st.n, paulis[t], flip[t], sign[t], q[t]);
    DeviceGuard g(st.device);
    expval_terms(st, flip, sign, q, out);
  });
}

KB_API int ketgpu_expval(const ketgpu_state* s, const char* pauli, double* out) {
  return guard([&] {
    need(s && out, "null argument");
    const State& st = *as_state(s);
    std::vector<uint64_t> flip(1), sign(1);
    std::vector<int> q(1);
    pauli_masks(st.n, pauli, flip[0], sign[0], q[0]);
    DeviceGuard g(st.device);
    expval_terms(st, flip, sign, q, out);
  });
}

KB_API int ketgpu_expval_sum(const ketgpu_state* s, const double* coeffs, const char* const* paulis,
                             uint64_t n_terms, double* out) {
  return guard([&] {
    need(s && out, "null argument");
    need((coeffs && paulis) || n_terms == 0, "null argument");
    const State& st = *as_state(s);
    std::vector<uint64_t> flip(n_terms), sign(n_terms);
    std::vector<int> q(n_terms);
    for (uint64_t t = 0; t < n_terms; ++t) pauli_masks(st.n, paulis[t], flip[t], sign[t], q[t]);
    std::vector<double> per(n_terms);
    DeviceGuard g(st.device);
    expval_terms(st, flip, sign, q, per.data());
    double total = 0.0;  // coefficient-weighted, in term order (observable.cpp:85-91)
    for (uint64_t t = 0; t < n_terms; ++t) total += coeffs[t] * per[t];
    *out = total;
  });
}

KB_API int ketgpu_uniforms_mt19937(uint32_t seed, uint64_t count, double* out) {
  return guard([&] {
    need(out != nullptr || count == 0, "out is null");
    std::mt19937 rng{seed};
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (uint64_t i = 0; i < count; ++i) out[i] = dist(rng);
  });
}

KB_API int ketgpu_sample(const ketgpu_state* s, const double* u, uint64_t count, uint64_t* out) {
  return guard([&] {
    need(s != nullptr, "state is null");
    need((u && out) || count == 0, "null argument");
    DeviceGuard g(as_state(s)->device);
    sample_tree(*as_state(s), u, count, out);
  });
}

KB_API int ketgpu_sample_seeded(const ketgpu_state* s, uint32_t seed, uint64_t count, uint64_t* out) {
  return guard([&] {
    need(s != nullptr, "state is null");
    need(out != nullptr || count == 0, "out is null");
    std::vector<double> u(count);
    std::mt19937 rng{seed};
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (uint64_t i = 0; i < count; ++i) u[i] = dist(rng);
    DeviceGuard g(as_state(s)->device);
    sample_tree(*as_state(s), u.data(), count, out);
  });
}

KB_API uint64_t ketgpu_sample_tree_builds(void) { return sample_tree_builds(); }

KB_API int ketgpu_measure(const ketgpu_state* s, uint32_t seed, uint64_t* out) {
  return guard([&] {
    need(s && out, "null argument");
    std::mt19937 rng{seed};
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    const double u = dist(rng);
    DeviceGuard g(as_state(s)->device);
    sample_tree(*as_state(s), &u, 1, out);
  });
}

KB_API int ketgpu_plan_execute_timed(const ketgpu_plan* p, ketgpu_state* s, float* pass_ms) {
  return guard([&] {
    need(p && s && pass_ms, "null argument");
    const Plan& plan = *as_plan(p);
    State& st = *as_state(s);
    need(plan.n == st.n && plan.precision == st.precision, "plan and state do not match");
    DeviceGuard g(st.device);
    upload_plan_matrices(const_cast<Plan&>(plan), st.device);
    const size_t np = plan.passes.size();
    std::vector<cudaEvent_t> ev(np + 1);
    for (auto& e : ev) KB_CUDA(cudaEventCreate(&e));
    KB_CUDA(cudaEventRecord(ev[0], st.stream));
    for (size_t i = 0; i < np; ++i) {
      launch_pass(st, plan, plan.passes[i]);
      KB_CUDA(cudaEventRecord(ev[i + 1], st.stream));
    }
    KB_CUDA(cudaEventSynchronize(ev[np]));
    for (size_t i = 0; i < np; ++i) KB_CUDA(cudaEventElapsedTime(&pass_ms[i], ev[i], ev[i + 1]));
    for (auto& e : ev) cudaEventDestroy(e);
    check_tc_flag();
  });
}

KB_API int ketgpu_plan_pass_info(const ketgpu_plan* p, uint64_t index, int32_t* kind, int32_t* k,
                                 int32_t* tensor, double* bytes) {
  return guard([&] {
    need(p != nullptr, "plan is null");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    if (kind)
      *kind = ps.kind == PassKind::Pair        ? 0
              : ps.kind == PassKind::Phase     ? 1
              : ps.kind == PassKind::Fused     ? 2
              : ps.kind == PassKind::Diagonal  ? 4
              : ps.kind == PassKind::SharedRun ? 5
                                               : 3;
    if (k)
      *k = (ps.kind == PassKind::Fused || ps.kind == PassKind::Diagonal) ? ps.k
           : ps.kind == PassKind::SharedRun                              ? ps.n_gates
                                                                         : ps.nfixed;
    if (tensor) *tensor = ps.tensor ? 1 : 0;
    if (bytes) *bytes = ps.bytes(plan.n, plan.precision == KETGPU_C64 ? 8 : 16);
  });
}

KB_API int ketgpu_plan_pass_qubits(const ketgpu_plan* p, uint64_t index, int32_t* qubits,
                                   int32_t capacity, int32_t* count) {
  return guard([&] {
    need(p != nullptr && count != nullptr, "null argument");
    need(capacity >= 0 && (capacity == 0 || qubits != nullptr), "bad qubit buffer");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    const int* q = nullptr;
    int nq = 0;
    if (ps.kind == PassKind::Fused) {
      q = ps.qubits;
      nq = ps.k;
    } else if (ps.kind == PassKind::Pair || ps.kind == PassKind::Phase) {
      q = ps.fixed;
      nq = ps.nfixed;
    }
    for (int i = 0; i < nq && i < capacity; ++i) qubits[i] = q[i];
    *count = nq;
  });
}

KB_API int ketgpu_plan_pass_gates(const ketgpu_plan* p, uint64_t index, int32_t* gates, int32_t capacity,
                                  int32_t* count) {
  return guard([&] {
    need(p != nullptr && count != nullptr, "null argument");
    need(capacity >= 0 && (capacity == 0 || gates != nullptr), "bad gate buffer");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    for (size_t i = 0; i < ps.gates.size() && (int32_t)i < capacity; ++i) gates[i] = ps.gates[i];
    *count = (int32_t)ps.gates.size();
  });
}

KB_API int ketgpu_plan_pass_tc_form(const ketgpu_plan* p, uint64_t index, int32_t* tma_dims, int32_t* direct) {
  return guard([&] {
    need(p != nullptr && tma_dims != nullptr && direct != nullptr, "null argument");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    if (ps.kind != PassKind::Fused || !ps.tensor) fail(KETGPU_ERR_INVALID, "pass is not a tensor-core block");
    int t = 0, d = 0;
    tc_form(plan.n, ps, &t, &d);
    *tma_dims = t;
    *direct = d;
  });
}

KB_API int ketgpu_plan_pass_matrix(const ketgpu_plan* p, uint64_t index, double* out, uint64_t capacity,
                                   uint64_t* count) {
  return guard([&] {
    need(p != nullptr && count != nullptr && (out != nullptr || capacity == 0), "null argument");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    if (ps.kind != PassKind::Fused) fail(KETGPU_ERR_INVALID, "pass is not a dense block");
    const std::vector<cplx>& m = plan.matrices[ps.mat_index];
    *count = 2 * m.size();
    const uint64_t nd = std::min<uint64_t>(capacity, 2 * m.size());
    for (uint64_t i = 0; i < nd; ++i) out[i] = (i & 1) ? m[i / 2].imag() : m[i / 2].real();
  });
}

KB_API int ketgpu_tc_image(int32_t k, const double* mat, uint32_t* out, uint64_t capacity, uint64_t* words) {
  return guard([&] {
    need(mat != nullptr && words != nullptr && (out != nullptr || capacity == 0), "null argument");
    if (!tc_supported(k)) fail(KETGPU_ERR_INVALID, "tensor-core blocks have k = 4, 5 or 6");
    const size_t dim = size_t{1} << k;
    std::vector<cplx> m(dim * dim);
    for (size_t i = 0; i < dim * dim; ++i) m[i] = cplx(mat[2 * i], mat[2 * i + 1]);
    std::vector<uint32_t> img;
    build_tc_image(m, k, img);
    *words = img.size();
    std::memcpy(out, img.data(), std::min<uint64_t>(capacity, img.size()) * sizeof(uint32_t));
  });
}

KB_API void* ketgpu_state_stream(const ketgpu_state* s) {
  return s ? reinterpret_cast<void*>(as_state(s)->stream) : nullptr;
}

KB_API int ketgpu_compare(const ketgpu_state* a, const ketgpu_state* b, double* out5) {
  return guard([&] {
    need(a && b && out5, "null argument");
    need(as_state(a)->n == as_state(b)->n, "states differ in size");
    DeviceGuard g(as_state(a)->device);
    compare_states(*as_state(a), *as_state(b), out5);
  });
}

KB_API int ketgpu_plan_pass_features(const ketgpu_plan* p, uint64_t index, float* out48) {
  return guard([&] {
    need(p && out48, "null argument");
    const Plan& plan = *as_plan(p);
    if (index >= plan.passes.size()) fail(KETGPU_ERR_OUT_OF_RANGE, "pass index out of range");
    const Pass& ps = plan.passes[index];
    std::vector<const ketgpu_op*> gs;
    std::vector<int> qs;
    for (int gi : ps.gates) {
      gs.push_back(&plan.ops[gi]);
      for (int j = 0; j < gate_arity(plan.ops[gi].type); ++j)
        if (std::find(qs.begin(), qs.end(), plan.ops[gi].q[j]) == qs.end()) qs.push_back(plan.ops[gi].q[j]);
    }
    const bool fused = ps.kind == PassKind::Fused || ps.gates.size() > 1;
    pass_features(plan.n, plan.precision, gs, qs, fused, ps.tensor, out48);
  });
}
