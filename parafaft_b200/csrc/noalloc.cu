// b200fft_c2c_noalloc: a batched C2C transform that allocates no memory.
//
// Who needs it: some callers cannot call cudaMalloc at the point where they
// transform. Typical cases are a host application that hands out all device
// memory itself from a pool fixed at start-up (so an extra library allocation
// can fail or break its accounting), and latency-critical loops that must not
// stall other streams: cudaMalloc and cudaFree may synchronize the device.
// A b200fft handle allocates a stream and a twiddle table, so those callers
// use this entry point instead.
//
// How: the one piece of memory the transform needs besides its input and
// output, the twiddle table, lives in a fixed array in the library's own
// device image (8192 complex doubles, 128 KiB, held on every device that loads
// the library until the process exits). Each call rewrites the table for its
// length in that array and then runs the specialised C2C kernel on the
// caller's stream; nothing in the array has to start at zero.
//
// Limits and rules for callers:
//  * lengths are powers of two from 2 to 4096 (the array's capacity); other
//    lengths are rejected with B200FFT_ERR_UNSUPPORTED before any GPU work;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture begins;
//  * the address is kept for the life of the process: calls after
//    cudaDeviceReset on that device are not supported (the module, and with
//    it the array, may move);
//  * the transform runs the specialised kernel's default tile (variant 0)
//    whatever the stride; a handle's plan may pick a wider column tile;
//  * every call on a device shares the one array and leaves its table there:
//    two calls that can run at the same time on the GPU (different streams
//    without ordering between them) race on it. Order them on one stream or
//    with events.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/b200fft.h"
#include "fft_common.hpp"
#include "launch.hpp"

namespace b200fft {
void set_error_text(const std::string &msg); // api.cu: text of b200fft_last_error()
}

#define NOALLOC_MAX_LENGTH 4096

// The twiddle table of b200fft_c2c_noalloc: 2 * NOALLOC_MAX_LENGTH complex
// doubles (128 KiB), room for the table pyramid of the longest length. Host
// code must not pass this name to a kernel: on the host it only stands for the
// symbol. The device address comes from cudaGetSymbolAddress (device_table
// below).
static __device__ __align__(256) unsigned char g_noalloc_table[2 * NOALLOC_MAX_LENGTH * 16];

namespace {

constexpr int kNoAllocMaxLength = NOALLOC_MAX_LENGTH;
constexpr int kMaxDevices = 64;

std::mutex g_mu;
void *g_table_addr[kMaxDevices] = {nullptr};

int fail(int code, const std::string &msg) {
  b200fft::set_error_text(msg);
  return code;
}

// Device address of g_noalloc_table on the current device, resolved once per
// device with that device current.
int device_table(void **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(B200FFT_ERR_NO_DEVICE,
                std::string("b200fft_c2c_noalloc: no usable current device: ") +
                    cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_table_addr[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_table);
    if (e != cudaSuccess || p == nullptr)
      return fail(B200FFT_ERR_CUDA,
                  std::string("b200fft_c2c_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
    g_table_addr[dev] = p;
  }
  *out = g_table_addr[dev];
  return B200FFT_SUCCESS;
}

} // namespace

extern "C" int b200fft_c2c_noalloc(int precision, int direction, int length, size_t batch,
                                   ptrdiff_t stride, ptrdiff_t dist, const void *in,
                                   void *out, void *cuda_stream) {
  using namespace b200fft;
  if (precision != B200FFT_F32 && precision != B200FFT_F64)
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft_c2c_noalloc: precision must be B200FFT_F32 or B200FFT_F64");
  if (direction != B200FFT_FORWARD && direction != B200FFT_BACKWARD)
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft_c2c_noalloc: direction must be B200FFT_FORWARD or B200FFT_BACKWARD");
  if (in == nullptr || out == nullptr || batch < 1 || stride < 1 || dist < 1)
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft_c2c_noalloc: null data pointer or batch/stride/dist below 1");
  if (length > kNoAllocMaxLength || !static_pow2_ok(length))
    return fail(B200FFT_ERR_UNSUPPORTED,
                "b200fft_c2c_noalloc: length " + std::to_string(length) +
                    " is not a power of two in [2, " + std::to_string(kNoAllocMaxLength) +
                    "] (the size of its fixed twiddle array)");
  if (batch > (1ull << 40) || stride > (1ll << 44) || dist > (1ll << 44))
    return fail(B200FFT_ERR_RANGE,
                "b200fft_c2c_noalloc: batch/stride/dist exceed the supported range");
  void *table = nullptr;
  int rc = device_table(&table);
  if (rc != B200FFT_SUCCESS)
    return rc;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  const bool f64 = precision == B200FFT_F64;
  // The whole table for this length is rewritten, so nothing left by an
  // earlier call is read.
  cudaError_t e = f64 ? launch_twiddle_table(static_cast<double2 *>(table), nullptr, length, st)
                      : launch_twiddle_table(nullptr, static_cast<float2 *>(table), length, st);
  if (e != cudaSuccess)
    return fail(B200FFT_ERR_CUDA,
                std::string("b200fft_c2c_noalloc: twiddle kernel: ") + cudaGetErrorString(e));
  PassArgs a{};
  a.in = in;
  a.out = out;
  a.tw = table;
  a.total = static_cast<long long>(batch);
  a.batch = static_cast<long long>(batch);
  a.idist = a.odist = dist;
  a.istride = a.ostride = stride;
  a.islab = a.oslab = 0;
  const bool col = dist < stride;
  const bool fwd = direction == B200FFT_FORWARD;
  e = f64 ? launch_static_c2c_f64(length, col, fwd, 0, a, st)
          : launch_static_c2c_f32(length, col, fwd, 0, a, st);
  if (e != cudaSuccess)
    return fail(B200FFT_ERR_CUDA,
                std::string("b200fft_c2c_noalloc: transform kernel: ") + cudaGetErrorString(e));
  return B200FFT_SUCCESS;
}
