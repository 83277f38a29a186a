// pack.cu - the 48-bit wire format of residues: each uint64 residue (< 2^47)
// travels as its 6 low bytes, little-endian, densely packed (25 % fewer bytes
// over PCIe than uint64 words).  One thread converts 8 words <-> 48 bytes
// (three 16-byte vectors), so a group always starts 16-byte aligned.
#include "dispatch.cuh"

__global__ void k_unpack48(u64* __restrict__ out, const unsigned char* __restrict__ in, long long n) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // group of 8 words
  const long long w0 = g * 8;
  if (w0 >= n) return;
  if (w0 + 8 <= n) {
    const uint4* src = reinterpret_cast<const uint4*>(in + g * 48);
    uint4 v[3] = {__ldg(src), __ldg(src + 1), __ldg(src + 2)};
    const unsigned char* b = reinterpret_cast<const unsigned char*>(v);
    u64 w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      u64 x = 0;
#pragma unroll
      for (int k = 5; k >= 0; --k) x = (x << 8) | b[6 * i + k];
      w[i] = x;
    }
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(out + w0);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = make_ulonglong2(w[2 * i], w[2 * i + 1]);
  } else {
    for (long long j = w0; j < n; ++j) {
      u64 x = 0;
      for (int k = 5; k >= 0; --k) x = (x << 8) | in[j * 6 + k];
      out[j] = x;
    }
  }
}

__global__ void k_pack48(unsigned char* __restrict__ out, const u64* __restrict__ in, long long n) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long w0 = g * 8;
  if (w0 >= n) return;
  if (w0 + 8 <= n) {
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(in + w0);
    u64 w[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const ulonglong2 p = src[i];
      w[2 * i] = p.x;
      w[2 * i + 1] = p.y;
    }
    uint4 v[3];
    unsigned char* b = reinterpret_cast<unsigned char*>(v);
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int k = 0; k < 6; ++k) b[6 * i + k] = (unsigned char)(w[i] >> (8 * k));
    uint4* dst = reinterpret_cast<uint4*>(out + g * 48);
    dst[0] = v[0];
    dst[1] = v[1];
    dst[2] = v[2];
  } else {
    for (long long j = w0; j < n; ++j)
      for (int k = 0; k < 6; ++k) out[j * 6 + k] = (unsigned char)(in[j] >> (8 * k));
  }
}

int ckks_launch_unpack48(uint64_t* out, const void* in, long long n, cudaStream_t st) {
  if (n <= 0) return CKKS_OK;
  k_unpack48<<<grid1d((n / 8 + 1 + 255) / 256), 256, 0, st>>>(reinterpret_cast<u64*>(out),
                                                              reinterpret_cast<const unsigned char*>(in), n);
  return ckks_check_launch("unpack48");
}

int ckks_launch_pack48(void* out, const uint64_t* in, long long n, cudaStream_t st) {
  if (n <= 0) return CKKS_OK;
  k_pack48<<<grid1d((n / 8 + 1 + 255) / 256), 256, 0, st>>>(reinterpret_cast<unsigned char*>(out),
                                                            reinterpret_cast<const u64*>(in), n);
  return ckks_check_launch("pack48");
}

extern "C" int ckks_unpack48(uint64_t* out, const void* in, long long n, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_unpack48: n < 0");
  CKKS_REQUIRE(n == 0 || (out && in), "ckks_unpack48: NULL pointer argument");
  CKKS_REQUIRE((reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0,
               "ckks_unpack48: buffers must be 16-byte aligned");
  return ckks_launch_unpack48(out, in, n, as_stream(stream));
}

extern "C" int ckks_pack48(void* out, const uint64_t* in, long long n, void* stream) {
  CKKS_REQUIRE(n >= 0, "ckks_pack48: n < 0");
  CKKS_REQUIRE(n == 0 || (out && in), "ckks_pack48: NULL pointer argument");
  CKKS_REQUIRE((reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0,
               "ckks_pack48: buffers must be 16-byte aligned");
  return ckks_launch_pack48(out, in, n, as_stream(stream));
}
