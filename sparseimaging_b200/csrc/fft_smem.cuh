// Shared-memory mixed-radix Stockham FFT, executed cooperatively by a CTA.
//
// `count` independent transforms of length n live in shared memory at
// data[t*ld + k]; every stage reads one buffer and writes the other
// (auto-sort, no bit reversal), so both buffers must hold count*ld values.
// Radices 4 and 2 cover powers of two; 3 and 5 have closed-form butterflies;
// any other prime factor (<= kMaxGenericRadix) uses a direct DFT.
// Forward sign is -1 (exp(-2 pi i jk/n)), unnormalised, matching FFTW's
// convention for the transforms the reference plans
// (c/mfista_nufft_lib.c:609-610, c/mfista_fft_lib.c:246-247).
#pragma once
#include "common.cuh"

namespace mf {

constexpr int kMaxGenericRadix = 16;

template <typename T>
__device__ __forceinline__ cplx<T> tw_get(const cplx<T>* __restrict__ tw, int idx, int sign) {
  cplx<T> w = tw[idx];
  return sign < 0 ? w : cconj<T>(w);
}

template <typename T>
__device__ __forceinline__ void bfly2(cplx<T>* v) {
  cplx<T> a = v[0], b = v[1];
  v[0] = cadd<T>(a, b);
  v[1] = csub<T>(a, b);
}

template <typename T>
__device__ __forceinline__ void bfly4(cplx<T>* v, int sign) {
  cplx<T> t0 = cadd<T>(v[0], v[2]), t1 = csub<T>(v[0], v[2]);
  cplx<T> t2 = cadd<T>(v[1], v[3]), t3 = cmul_si<T>(csub<T>(v[1], v[3]), sign);
  v[0] = cadd<T>(t0, t2);
  v[2] = csub<T>(t0, t2);
  v[1] = cadd<T>(t1, t3);
  v[3] = csub<T>(t1, t3);
}

template <typename T>
__device__ __forceinline__ void bfly3(cplx<T>* v, int sign) {
  const T c3 = T(-0.5), s3 = T(0.86602540378443864676);
  cplx<T> t1 = cadd<T>(v[1], v[2]);
  cplx<T> t2 = csub<T>(v[1], v[2]);
  cplx<T> m1 = mk<T>(v[0].x + c3 * t1.x, v[0].y + c3 * t1.y);
  cplx<T> m2 = cmul_si<T>(mk<T>(s3 * t2.x, s3 * t2.y), sign);
  v[0] = cadd<T>(v[0], t1);
  v[1] = cadd<T>(m1, m2);
  v[2] = csub<T>(m1, m2);
}

template <typename T>
__device__ __forceinline__ void bfly5(cplx<T>* v, int sign) {
  const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
  const T s1 = T(0.95105651629515357212), s2 = T(0.58778525229247312917);
  cplx<T> a1 = cadd<T>(v[1], v[4]), b1 = csub<T>(v[1], v[4]);
  cplx<T> a2 = cadd<T>(v[2], v[3]), b2 = csub<T>(v[2], v[3]);
  cplx<T> r1 = mk<T>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
  cplx<T> r2 = mk<T>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
  cplx<T> i1 = cmul_si<T>(mk<T>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), sign);
  cplx<T> i2 = cmul_si<T>(mk<T>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), sign);
  v[0] = mk<T>(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
  v[1] = cadd<T>(r1, i1);
  v[4] = csub<T>(r1, i1);
  v[2] = cadd<T>(r2, i2);
  v[3] = csub<T>(r2, i2);
}

// One radix-R stage over all `count` transforms.  Returns nothing; caller syncs.
template <typename T, int R>
__device__ __forceinline__ void stockham_stage(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst,
                                               int n, int ld, int count, int Ns, const cplx<T>* __restrict__ tw,
                                               int sign) {
  const int nR = n / R;
  const int tstride = n / (Ns * R);
  // powers of two (the usual grid sizes): the index arithmetic as shifts and
  // masks instead of integer divisions (the same indices)
  const bool pow2 = ((nR & (nR - 1)) == 0) && ((Ns & (Ns - 1)) == 0);
  const int lnR = __ffs(nR) - 1, lNs = __ffs(Ns) - 1;
  for (int t = threadIdx.x; t < count * nR; t += blockDim.x) {
    int tr, j, k, jq;
    if (pow2) {
      tr = t >> lnR;
      j = t & (nR - 1);
      k = j & (Ns - 1);
      jq = j >> lNs;
    } else {
      tr = t / nR;
      j = t - tr * nR;
      k = j % Ns;
      jq = j / Ns;
    }
    const cplx<T>* s = src + (size_t)tr * ld;
    cplx<T>* d = dst + (size_t)tr * ld;
    cplx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cplx<T> a = s[j + r * nR];
      if (r > 0 && k > 0) a = cmul<T>(a, tw_get<T>(tw, k * r * tstride, sign));
      v[r] = a;
    }
    if (R == 2) bfly2<T>(v);
    else if (R == 4) bfly4<T>(v, sign);
    else if (R == 3) bfly3<T>(v, sign);
    else if (R == 5) bfly5<T>(v, sign);
    int base = jq * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[base + r * Ns] = v[r];
  }
}

template <typename T>
__device__ void stockham_stage_generic(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, int n, int ld,
                                       int count, int Ns, int R, const cplx<T>* __restrict__ tw, int sign) {
  const int nR = n / R;
  const int tstride = n / (Ns * R);
  const int step = n / R;
  for (int t = threadIdx.x; t < count * nR; t += blockDim.x) {
    int tr = t / nR;
    int j = t - tr * nR;
    int k = j % Ns;
    const cplx<T>* s = src + (size_t)tr * ld;
    cplx<T>* d = dst + (size_t)tr * ld;
    cplx<T> v[kMaxGenericRadix];
    for (int r = 0; r < R; ++r) {
      cplx<T> a = s[j + r * nR];
      if (r > 0 && k > 0) a = cmul<T>(a, tw_get<T>(tw, k * r * tstride, sign));
      v[r] = a;
    }
    int base = (j / Ns) * Ns * R + k;
    for (int q = 0; q < R; ++q) {
      cplx<T> acc = v[0];
      for (int r = 1; r < R; ++r) acc = cadd<T>(acc, cmul<T>(v[r], tw_get<T>(tw, ((r * q) % R) * step, sign)));
      d[base + q * Ns] = acc;
    }
  }
}

// Runs all stages.  Input in `a`; returns the buffer holding the result
// (a or b).  Ends with a __syncthreads().
template <typename T>
__device__ cplx<T>* smem_fft(cplx<T>* a, cplx<T>* b, const FftDev<T>& p, int ld, int count, int sign) {
  cplx<T>* src = a;
  cplx<T>* dst = b;
  int Ns = 1;
  for (int s = 0; s < p.nst; ++s) {
    int R = p.radix[s];
    switch (R) {
      case 4: stockham_stage<T, 4>(src, dst, p.n, ld, count, Ns, p.tw, sign); break;
      case 2: stockham_stage<T, 2>(src, dst, p.n, ld, count, Ns, p.tw, sign); break;
      case 3: stockham_stage<T, 3>(src, dst, p.n, ld, count, Ns, p.tw, sign); break;
      case 5: stockham_stage<T, 5>(src, dst, p.n, ld, count, Ns, p.tw, sign); break;
      default: stockham_stage_generic<T>(src, dst, p.n, ld, count, Ns, R, p.tw, sign); break;
    }
    __syncthreads();
    cplx<T>* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace mf
