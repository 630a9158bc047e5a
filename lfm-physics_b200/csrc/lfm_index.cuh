// Periodic 19-point neighbourhood of a cell in a flat (N, N, N) C-order
// lattice: the offsets np.roll reaches in lfm/core/stencils.py:43-71.
#pragma once

#include <cstdint>

#include "lfm_math.cuh"

namespace lfm {

struct Idx {
  int64_t c, im, ip, jm, jp, km, kp;
  int64_t imjm, imjp, ipjm, ipjp, imkm, imkp, ipkm, ipkp, jmkm, jmkp, jpkm, jpkp;
};

__device__ __forceinline__ Idx neighbour_index(int i, int j, int k, int N) {
  const int64_t n = N;
  const int64_t im = (i == 0 ? N - 1 : i - 1), ip = (i == N - 1 ? 0 : i + 1);
  const int64_t jm = (j == 0 ? N - 1 : j - 1), jp = (j == N - 1 ? 0 : j + 1);
  const int64_t km = (k == 0 ? N - 1 : k - 1), kp = (k == N - 1 ? 0 : k + 1);
  const int64_t I0 = im * n * n, I1 = (int64_t)i * n * n, I2 = ip * n * n;
  const int64_t J0 = jm * n, J1 = (int64_t)j * n, J2 = jp * n;
  Idx x;
  x.c = I1 + J1 + k;
  x.im = I0 + J1 + k;   x.ip = I2 + J1 + k;
  x.jm = I1 + J0 + k;   x.jp = I1 + J2 + k;
  x.km = I1 + J1 + km;  x.kp = I1 + J1 + kp;
  x.imjm = I0 + J0 + k; x.imjp = I0 + J2 + k; x.ipjm = I2 + J0 + k; x.ipjp = I2 + J2 + k;
  x.imkm = I0 + J1 + km; x.imkp = I0 + J1 + kp; x.ipkm = I2 + J1 + km; x.ipkp = I2 + J1 + kp;
  x.jmkm = I1 + J0 + km; x.jmkp = I1 + J0 + kp; x.jpkm = I1 + J2 + km; x.jpkp = I1 + J2 + kp;
  return x;
}

// The same neighbourhood in a slab array: planes i-1 and i+1 are read as they
// are (ghost planes hold the neighbours' data), j and k wrap.
__device__ __forceinline__ Idx neighbour_index_slab(int i, int j, int k, int N) {
  const int64_t n = N;
  const int64_t im = i - 1, ip = i + 1;
  const int64_t jm = (j == 0 ? N - 1 : j - 1), jp = (j == N - 1 ? 0 : j + 1);
  const int64_t km = (k == 0 ? N - 1 : k - 1), kp = (k == N - 1 ? 0 : k + 1);
  const int64_t I0 = im * n * n, I1 = (int64_t)i * n * n, I2 = ip * n * n;
  const int64_t J0 = jm * n, J1 = (int64_t)j * n, J2 = jp * n;
  Idx x;
  x.c = I1 + J1 + k;
  x.im = I0 + J1 + k;   x.ip = I2 + J1 + k;
  x.jm = I1 + J0 + k;   x.jp = I1 + J2 + k;
  x.km = I1 + J1 + km;  x.kp = I1 + J1 + kp;
  x.imjm = I0 + J0 + k; x.imjp = I0 + J2 + k; x.ipjm = I2 + J0 + k; x.ipjp = I2 + J2 + k;
  x.imkm = I0 + J1 + km; x.imkp = I0 + J1 + kp; x.ipkm = I2 + J1 + km; x.ipkp = I2 + J1 + kp;
  x.jmkm = I1 + J0 + km; x.jmkp = I1 + J0 + kp; x.jpkm = I1 + J2 + km; x.jpkp = I1 + J2 + kp;
  return x;
}

__device__ __forceinline__ S19 gather(const float* __restrict__ f, const Idx& x) {
  S19 s;
  s.c = __ldg(f + x.c);
  s.im = __ldg(f + x.im); s.ip = __ldg(f + x.ip);
  s.jm = __ldg(f + x.jm); s.jp = __ldg(f + x.jp);
  s.km = __ldg(f + x.km); s.kp = __ldg(f + x.kp);
  s.imjm = __ldg(f + x.imjm); s.imjp = __ldg(f + x.imjp);
  s.ipjm = __ldg(f + x.ipjm); s.ipjp = __ldg(f + x.ipjp);
  s.imkm = __ldg(f + x.imkm); s.imkp = __ldg(f + x.imkp);
  s.ipkm = __ldg(f + x.ipkm); s.ipkp = __ldg(f + x.ipkp);
  s.jmkm = __ldg(f + x.jmkm); s.jmkp = __ldg(f + x.jmkp);
  s.jpkm = __ldg(f + x.jpkm); s.jpkp = __ldg(f + x.jpkp);
  return s;
}

}  // namespace lfm
