// ref_spectral_host.cu -- host launcher for the reference's own CUDA sieve kernel
// (spectral_scan_kernel, src/cuda/spectral.cu:136-213 of kira-ls-aligner), which
// this recipe compiles from the reference source tree for sm_100a. TEST
// INFRASTRUCTURE ONLY: a second parity pin for the sieve and a timing comparator.
//
// The launcher reproduces CudaBackend::run_batch (src/cuda/backend.rs:95-249):
// reads padded to 64 bytes, the window's four bit phases concatenated
// phase-major, sentinel-initialised outputs, grid = n, block = 32.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "spectral.cu"  // the reference kernel, from -I<reference>/src/cuda

namespace {
constexpr int kReadBytesMax = 64;

void shift_right(const uint8_t* bits, size_t n, int off, uint8_t* out) {
  if (off == 0) {
    if (n) std::memcpy(out, bits, n);
    return;
  }
  for (size_t i = 0; i < n; ++i)
    out[i] = (uint8_t)((bits[i] >> off) | (i + 1 < n ? (uint8_t)(bits[i + 1] << (8 - off)) : 0));
}
}  // namespace

extern "C" {

// jobs: packed reads (read_off/read_bytes into reads), packed phase-0 windows
// (ref_off/ref_bytes into refs). Returns 0 on success; kernel_ms receives the
// kernel time (CUDA events), total_ms the whole run_batch time (H2D+kernel+D2H).
int ref_spectral_run_batch(int n, const uint8_t* reads, const uint64_t* read_off,
                           const uint32_t* read_bytes, const uint32_t* read_nucs,
                           const uint8_t* refs, const uint64_t* ref_off,
                           const uint32_t* ref_bytes, const uint32_t* ref_nucs,
                           const uint32_t* max_mism, int32_t* out_shift, int32_t* out_mism,
                           int32_t* out_second, float* kernel_ms, float* total_ms) {
  if (n <= 0) return 0;
  cudaEvent_t t0, t1, k0, k1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  cudaEventRecord(t0);
  std::vector<uint8_t> hreads((size_t)n * kReadBytesMax, 0);
  std::vector<int32_t> hrl(n), hoff(n), hlen(n), hlim(n);
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    if (read_bytes[i] > (uint32_t)kReadBytesMax) return 5;
    std::memcpy(&hreads[(size_t)i * kReadBytesMax], reads + read_off[i], read_bytes[i]);
    hrl[i] = (int32_t)read_nucs[i];
    total += ref_bytes[i];
  }
  std::vector<uint8_t> flat(4 * total + 1, 0);
  size_t acc = 0;
  for (int i = 0; i < n; ++i) {
    for (int ph = 0; ph < 4; ++ph)
      shift_right(refs + ref_off[i], ref_bytes[i], 2 * ph, flat.data() + ph * total + acc);
    hoff[i] = (int32_t)acc;
    hlen[i] = (int32_t)ref_nucs[i];
    hlim[i] = (int32_t)std::min(max_mism[i], read_nucs[i]);
    acc += ref_bytes[i];
  }
  std::vector<int32_t> init_s(n, -1), init_m(2 * (size_t)n, INT32_MAX);
  uint8_t *dr = nullptr, *df = nullptr;
  int32_t *drl = nullptr, *doff = nullptr, *dlen = nullptr, *dlim = nullptr, *ds = nullptr,
          *dm = nullptr;
  cudaMalloc(&dr, hreads.size());
  cudaMalloc(&df, flat.size());
  cudaMalloc(&drl, 4 * n);
  cudaMalloc(&doff, 4 * n);
  cudaMalloc(&dlen, 4 * n);
  cudaMalloc(&dlim, 4 * n);
  cudaMalloc(&ds, 4 * n);
  cudaMalloc(&dm, 8 * (size_t)n);
  cudaMemcpy(dr, hreads.data(), hreads.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(df, flat.data(), flat.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(drl, hrl.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(doff, hoff.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dlen, hlen.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dlim, hlim.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(ds, init_s.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dm, init_m.data(), 8 * (size_t)n, cudaMemcpyHostToDevice);
  cudaEventRecord(k0);
  spectral_scan_kernel<<<n, 32>>>(dr, drl, df, (int32_t)total, doff, dlen, kReadBytesMax, dlim, n,
                                  ds, dm);
  cudaEventRecord(k1);
  std::vector<int32_t> hm(2 * (size_t)n);
  cudaMemcpy(out_shift, ds, 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(hm.data(), dm, 8 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  const cudaError_t err = cudaGetLastError();
  for (int i = 0; i < n; ++i) {
    out_mism[i] = hm[i];
    out_second[i] = hm[(size_t)n + i];
  }
  cudaEventElapsedTime(kernel_ms, k0, k1);
  cudaEventElapsedTime(total_ms, t0, t1);
  cudaFree(dr);
  cudaFree(df);
  cudaFree(drl);
  cudaFree(doff);
  cudaFree(dlen);
  cudaFree(dlim);
  cudaFree(ds);
  cudaFree(dm);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(k0);
  cudaEventDestroy(k1);
  return err == cudaSuccess ? 0 : 3;
}
}
