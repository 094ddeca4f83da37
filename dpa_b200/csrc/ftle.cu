// ftle.cu -- flow-map scatter, central-difference Jacobian, C = J^T J,
// FP64 largest eigenvalue and ln(sqrt(lambda)) / T per lattice cell
// (ftle_estimator.cpp:7-65 with regular_grid::gradient, regular_grid.hpp:87-108).
#include "kernels.cuh"

namespace dpa {

namespace {

inline unsigned blocks_for(uint64_t n, unsigned block) { return unsigned((n + block - 1) / block); }

__device__ __forceinline__ bool reference_cell(const FtleArgs& a, uint64_t p, uint64_t& cell) {
  uint64_t sub[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    // regular_grid::cell_index (regular_grid.hpp:28-34) on the flow map.
    const float s = floorf(__fdiv_rn(__fsub_rn(a.original_positions[3 * p + i], a.offset[i]),
                                     a.spacing[i]));
    if (!(s >= 0.0f) || !(s < float(a.shape[i]))) return false;
    sub[i] = uint64_t(s);
  }
  cell = (sub[0] * a.shape[1] + sub[1]) * a.shape[2] + sub[2];
  return true;
}

// Pass 1: every particle claims its cell; the largest particle index wins.
__global__ void ftle_claim_kernel(const FtleArgs a) {
  const uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= a.count) return;
  uint64_t cell;
  if (reference_cell(a, p, cell)) atomicMax(a.winners + cell, (unsigned long long)(p + 1));
}

// Pass 2: the flow map holds the winner's final position, zero where no
// particle landed (the reference's zero-initialized multi_array).
__global__ void ftle_fill_kernel(const FtleArgs a, uint64_t cells) {
  const uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  float x = 0.0f, y = 0.0f, z = 0.0f;
  if (a.mapping == DPA_FTLE_MAPPING_LATTICE) {
    x = a.final_positions[3 * c];
    y = a.final_positions[3 * c + 1];
    z = a.final_positions[3 * c + 2];
  } else {
    const unsigned long long w = a.winners[c];
    if (w) {
      const uint64_t p = w - 1;
      x = a.final_positions[3 * p];
      y = a.final_positions[3 * p + 1];
      z = a.final_positions[3 * p + 2];
    }
  }
  a.flow[3 * c] = x;
  a.flow[3 * c + 1] = y;
  a.flow[3 * c + 2] = z;
}

// Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations.
__device__ double max_eigenvalue(double a[3][3]) {
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off == 0.0 || off <= 1e-32 * diag) break;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
#pragma unroll
      for (int q = p + 1; q < 3; ++q) {
        const double apq = a[p][q];
        if (apq == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double arp = a[r][p], arq = a[r][q];
          a[r][p] = c * arp - s * arq;
          a[r][q] = s * arp + c * arq;
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double apr = a[p][r], aqr = a[q][r];
          a[p][r] = c * apr - s * aqr;
          a[q][r] = s * apr + c * aqr;
        }
      }
    }
  }
  return fmax(a[0][0], fmax(a[1][1], a[2][2]));
}

// Pass 3: per lattice cell. J[r][d] = (flow[next_d] - flow[prev_d])[r] / (2 h_d)
// with prev/next clamped at the border while the divisor stays 2 h_d.
// C = J^T J in FP32 (Eigen's 3x3 lazy product, c0 + (c1 + c2)); the
// eigenvalue and the logarithm in FP64.
__global__ void ftle_kernel(const FtleArgs a, uint64_t cells) {
  const uint64_t flat = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (flat >= cells) return;
  const uint64_t n1n2 = a.shape[1] * a.shape[2];
  uint64_t sub[3] = {flat / n1n2, (flat / a.shape[2]) % a.shape[1], flat % a.shape[2]};
  const uint64_t step[3] = {n1n2, a.shape[2], 1};
  float J[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const uint64_t prev = sub[d] > 0 ? flat - step[d] : flat;
    const uint64_t next = sub[d] + 1 < a.shape[d] ? flat + step[d] : flat;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      J[r][d] = __fdiv_rn(__fsub_rn(a.flow[3 * next + r], a.flow[3 * prev + r]), a.two_spacing[d]);
  }
  double C[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      C[i][j] = double(__fadd_rn(__fmul_rn(J[0][i], J[0][j]),
                                 __fadd_rn(__fmul_rn(J[1][i], J[1][j]), __fmul_rn(J[2][i], J[2][j]))));
  const double lambda = max_eigenvalue(C);
  a.ftle[flat] = float(log(sqrt(lambda)) / a.horizon);
}

__global__ void lattice_kernel(float o0, float o1, float o2, float s0, float s1, float s2,
                               uint64_t n0, uint64_t n1, uint64_t n2, float* out) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t count = n0 * n1 * n2;
  if (t >= count) return;
  // unravel_index (indexing.hpp:11-20): last axis fastest.
  const uint64_t i2 = t % n2, i1 = (t / n2) % n1, i0 = t / (n1 * n2);
  out[3 * t] = __fadd_rn(o0, __fmul_rn(s0, float(i0)));
  out[3 * t + 1] = __fadd_rn(o1, __fmul_rn(s1, float(i1)));
  out[3 * t + 2] = __fadd_rn(o2, __fmul_rn(s2, float(i2)));
}

// Counter-based seed stream: splitmix64 (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", 2014) of key ^ (3 i + axis).
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

__global__ void random_seeds_kernel(float o0, float o1, float o2, float s0, float s1, float s2,
                                    uint64_t count, uint64_t key, float* out) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const float o[3] = {o0, o1, o2}, s[3] = {s0, s1, s2};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const uint64_t r = splitmix64(key ^ (3 * t + uint64_t(a)));
    const float u = float(uint32_t(r >> 40)) * 0x1p-24f;  // [0, 1), 24 random bits
    out[3 * t + a] = __fadd_rn(o[a], __fmul_rn(s[a], u));
  }
}

}  // namespace

cudaError_t launch_random_seeds(const float offset[3], const float size[3], uint64_t count,
                                uint64_t key, float* out, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  random_seeds_kernel<<<blocks_for(count, 256), 256, 0, stream>>>(
      offset[0], offset[1], offset[2], size[0], size[1], size[2], count, key, out);
  return cudaGetLastError();
}

cudaError_t launch_ftle(const FtleArgs& a, cudaStream_t stream) {
  const uint64_t cells = a.shape[0] * a.shape[1] * a.shape[2];
  if (cells == 0) return cudaSuccess;
  if (a.mapping == DPA_FTLE_MAPPING_REFERENCE) {
    DPA_CUDA_TRY(cudaMemsetAsync(a.winners, 0, cells * sizeof(unsigned long long), stream));
    if (a.count) {
      ftle_claim_kernel<<<blocks_for(a.count, 256), 256, 0, stream>>>(a);
      DPA_CUDA_TRY(cudaGetLastError());
    }
  }
  ftle_fill_kernel<<<blocks_for(cells, 256), 256, 0, stream>>>(a, cells);
  DPA_CUDA_TRY(cudaGetLastError());
  ftle_kernel<<<blocks_for(cells, 128), 128, 0, stream>>>(a, cells);
  return cudaGetLastError();
}

cudaError_t launch_lattice_seeds(const float offset[3], const float stride[3],
                                 const uint64_t shape[3], float* out, cudaStream_t stream) {
  const uint64_t count = shape[0] * shape[1] * shape[2];
  if (count == 0) return cudaSuccess;
  lattice_kernel<<<blocks_for(count, 256), 256, 0, stream>>>(
      offset[0], offset[1], offset[2], stride[0], stride[1], stride[2], shape[0], shape[1],
      shape[2], out);
  return cudaGetLastError();
}

}  // namespace dpa
