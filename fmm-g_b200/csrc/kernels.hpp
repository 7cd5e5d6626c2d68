// kernels.hpp -- the kernel library of the reference (fmm3d_mpi/kernel3d_mpi.cpp:35-466)
// as header-only functors shared by the host operator builder and the CUDA
// stage kernels.  Each functor evaluates one (target, source) block
// K[t*SD + s] of the reference buildKnlIntCtx matrix for the offset
// (x, y, z) = target - source; a block with r < 1e-8 is zero
// (kernel3d_mpi.cpp:35, 160).
#pragma once

#include <cmath>
#include <type_traits>

#if defined(__CUDACC__)
#define FMMG_HD __host__ __device__ __forceinline__
#define FMMG_UNROLL _Pragma("unroll")
#else
#define FMMG_HD inline
#define FMMG_UNROLL
#endif

namespace fmmg {

enum KernelId {
  LAP_S_U = 111, LAP_D_U = 121, STK_F_U = 301, STK_S_U = 311, STK_S_P = 312,
  STK_D_U = 321, STK_D_P = 322, NAV_S_U = 511, NAV_D_U = 521
};

// DOFs (kernel3d_mpi.cpp:40-103), whether the source normal enters, and the
// equivalent-density kernel setup() pairs with it (fmm3d_setup_mpi.cpp:113-126).
template <int KT> struct KTraits;
template <> struct KTraits<LAP_S_U> { enum { SD = 1, TD = 1, NRM = 0, MM = LAP_S_U }; };
template <> struct KTraits<LAP_D_U> { enum { SD = 1, TD = 1, NRM = 1, MM = LAP_S_U }; };
template <> struct KTraits<STK_F_U> { enum { SD = 4, TD = 3, NRM = 0, MM = STK_F_U }; };
template <> struct KTraits<STK_S_U> { enum { SD = 3, TD = 3, NRM = 0, MM = STK_F_U }; };
template <> struct KTraits<STK_S_P> { enum { SD = 3, TD = 1, NRM = 0, MM = LAP_S_U }; };
template <> struct KTraits<STK_D_U> { enum { SD = 3, TD = 3, NRM = 1, MM = STK_F_U }; };
template <> struct KTraits<STK_D_P> { enum { SD = 3, TD = 1, NRM = 1, MM = LAP_S_U }; };
template <> struct KTraits<NAV_S_U> { enum { SD = 3, TD = 3, NRM = 0, MM = NAV_S_U }; };
template <> struct KTraits<NAV_D_U> { enum { SD = 3, TD = 3, NRM = 1, MM = NAV_S_U }; };

inline int kernel_src_dof(int kt) {
  switch (kt) {
    case LAP_S_U: case LAP_D_U: return 1;
    case STK_F_U: return 4;
    case STK_S_U: case STK_S_P: case STK_D_U: case STK_D_P: case NAV_S_U: case NAV_D_U: return 3;
  }
  return 0;
}
inline int kernel_trg_dof(int kt) {
  switch (kt) {
    case LAP_S_U: case LAP_D_U: case STK_S_P: case STK_D_P: return 1;
    case STK_F_U: case STK_S_U: case STK_D_U: case NAV_S_U: case NAV_D_U: return 3;
  }
  return 0;
}
constexpr int kernel_mm(int kt) {
  switch (kt) {
    case LAP_S_U: case LAP_D_U: case STK_S_P: case STK_D_P: return LAP_S_U;
    case STK_S_U: case STK_D_U: return STK_F_U;
    case NAV_S_U: case NAV_D_U: return NAV_S_U;
  }
  return -1;
}
inline bool kernel_has_normal(int kt) {
  return kt == LAP_D_U || kt == STK_D_U || kt == STK_D_P || kt == NAV_D_U;
}
// homogeneous degree per source component (kernel3d_mpi.cpp:122-131)
inline int kernel_hom_deg(int kt, double* deg) {
  switch (kt) {
    case LAP_S_U: deg[0] = 1; return 1;
    case STK_F_U: deg[0] = deg[1] = deg[2] = 1; deg[3] = 2; return 4;
    case NAV_S_U: deg[0] = deg[1] = deg[2] = 1; return 3;
  }
  return 0;
}

template <typename R> FMMG_HD R fmmg_rsqrt(R v);
template <> FMMG_HD double fmmg_rsqrt<double>(double v) {
#if defined(__CUDA_ARCH__)
  return rsqrt(v);
#else
  return 1.0 / std::sqrt(v);
#endif
}
template <> FMMG_HD float fmmg_rsqrt<float>(float v) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(v);
#else
  return 1.0f / std::sqrt(v);
#endif
}

struct KCoef {
  double mu, ve;
};

// One block.  Returns false (block left unset) for a coincident pair.  For
// the double-layer kernels rnp, when given, holds (x, y, z) . n computed by
// the caller (the FP32 near field forms it in FP64: for close points on a
// smooth surface it is O(r^2) while its FP32 rounding error is O(eps r)).
template <int KT, typename R>
FMMG_HD bool kblock(R x, R y, R z, const R* n, R* K, R mu, R ve, const R* rnp = nullptr) {
  const R r2 = x * x + y * y + z * z;
  if (r2 < R(1e-16)) return false;
  const R ir = fmmg_rsqrt<R>(r2);
  const R ir3 = ir * ir * ir;
  const R PI = R(3.14159265358979323846);
  if constexpr (KT == LAP_S_U) {  // :152-167
    K[0] = R(1) / (R(4) * PI) * ir;
  } else if constexpr (KT == LAP_D_U) {  // :169-185
    R rn = rnp ? *rnp : x * n[0] + y * n[1] + z * n[2];
    K[0] = -(R(1) / (R(4) * PI)) * ir3 * rn;
  } else if constexpr (KT == STK_F_U) {  // :194-219
    R oomu = R(1) / mu;
    R G = oomu * (R(1) / (R(8) * PI)) * ir, H = oomu * (R(1) / (R(8) * PI)) * ir3;
    R A = (R(1) / (R(4) * PI)) * ir3;
    K[0] = G + H * x * x; K[1] = H * x * y; K[2] = H * x * z; K[3] = A * x;
    K[4] = H * y * x; K[5] = G + H * y * y; K[6] = H * y * z; K[7] = A * y;
    K[8] = H * z * x; K[9] = H * z * y; K[10] = G + H * z * z; K[11] = A * z;
  } else if constexpr (KT == STK_S_U || KT == NAV_S_U) {  // :221-242, :362-385
    R oomu = R(1) / mu;
    R G, H;
    if constexpr (KT == STK_S_U) {
      G = (R(1) / (R(8) * PI)) * ir;
      H = (R(1) / (R(8) * PI)) * ir3;
    } else {
      G = (R(3) - R(4) * ve) / (R(16) * PI * (R(1) - ve)) * ir;
      H = R(1) / (R(16) * PI * (R(1) - ve)) * ir3;
    }
    K[0] = oomu * (G + H * x * x); K[1] = oomu * (H * x * y); K[2] = oomu * (H * x * z);
    K[3] = oomu * (H * y * x); K[4] = oomu * (G + H * y * y); K[5] = oomu * (H * y * z);
    K[6] = oomu * (H * z * x); K[7] = oomu * (H * z * y); K[8] = oomu * (G + H * z * z);
  } else if constexpr (KT == STK_S_P) {  // :244-260
    R c = (R(1) / (R(4) * PI)) * ir3;
    K[0] = c * x; K[1] = c * y; K[2] = c * z;
  } else if constexpr (KT == STK_D_U) {  // :262-283
    R rn = rnp ? *rnp : x * n[0] + y * n[1] + z * n[2];
    R C = -(R(6) / (R(8) * PI)) * ir3 * ir * ir * rn;
    K[0] = C * x * x; K[1] = C * x * y; K[2] = C * x * z;
    K[3] = C * y * x; K[4] = C * y * y; K[5] = C * y * z;
    K[6] = C * z * x; K[7] = C * z * y; K[8] = C * z * z;
  } else if constexpr (KT == STK_D_P) {  // :285-308
    R rn = rnp ? *rnp : x * n[0] + y * n[1] + z * n[2];
    R c = mu * (R(1) / (R(2) * PI));
    R ir5 = ir3 * ir * ir;
    K[0] = c * (n[0] * ir3 - R(3) * rn * x * ir5);
    K[1] = c * (n[1] * ir3 - R(3) * rn * y * ir5);
    K[2] = c * (n[2] * ir3 - R(3) * rn * z * ir5);
  } else if constexpr (KT == NAV_D_U) {  // :387-419
    R rn = rnp ? *rnp : x * n[0] + y * n[1] + z * n[2];
    R A = -(R(1) - R(2) * ve) / (R(8) * PI * (R(1) - ve)) * ir3;
    R B = (R(1) - R(2) * ve) / (R(8) * PI * (R(1) - ve)) * ir3;
    R C = R(-3) / (R(8) * PI * (R(1) - ve)) * ir3 * ir * ir * rn;
    const R d[3] = {x, y, z};
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        K[a * 3 + b] = A * ((a == b ? rn : R(0)) + n[a] * d[b]) + B * (d[a] * n[b]) + C * d[a] * d[b];
  }
  return true;
}

// acc[t] += sum_s K[t][s] den[s]
template <int KT, typename R, typename A>
FMMG_HD void kaccum(R x, R y, R z, const R* n, const R* den, A* acc, R mu, R ve) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  R K[SD * TD];
  if (!kblock<KT, R>(x, y, z, n, K, mu, ve)) return;
FMMG_UNROLL
  for (int t = 0; t < TD; t++) {
    R s = R(0);
FMMG_UNROLL
    for (int c = 0; c < SD; c++) s += K[t * SD + c] * den[c];
    acc[t] += s;
  }
}

// KB right-hand sides at once: acc[r*TD + t] += sum_s K[t][s] den[r*SD + s];
// the kernel block is evaluated once and applied to every density.
template <int KT, int KB, typename R, typename A>
FMMG_HD void kaccum_multi(R x, R y, R z, const R* n, const R* den, A* acc, R mu, R ve, const R* rnp = nullptr) {
  constexpr int SD = KTraits<KT>::SD, TD = KTraits<KT>::TD;
  R K[SD * TD];
  if (!kblock<KT, R>(x, y, z, n, K, mu, ve, rnp)) return;
#if defined(__CUDA_ARCH__)
  if constexpr (SD == 1 && TD == 1 && KB % 2 == 0 && std::is_same<R, float>::value &&
                std::is_same<A, float>::value) {
    // scalar FP32 kernels: two right-hand sides per packed FP32x2 FMA (one
    // rounding per component, as fmaf(K, den, acc))
    unsigned long long kk;
    asm("mov.b64 %0, {%1, %1};" : "=l"(kk) : "f"(K[0]));
FMMG_UNROLL
    for (int r = 0; r < KB; r += 2) {
      unsigned long long a, d;
      asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(acc[r]), "f"(acc[r + 1]));
      asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(den[r]), "f"(den[r + 1]));
      asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(a) : "l"(kk), "l"(d));
      asm("mov.b64 {%0, %1}, %2;" : "=f"(acc[r]), "=f"(acc[r + 1]) : "l"(a));
    }
  } else
#endif
  {
FMMG_UNROLL
    for (int r = 0; r < KB; r++)
FMMG_UNROLL
      for (int t = 0; t < TD; t++) {
        // the first product starts the sum: an explicit 0 + x cannot be
        // dropped under IEEE rules and would cost an add per term (with SD = 1
        // the product and the accumulate fuse into one FMA)
        R s = K[t * SD] * den[r * SD];
FMMG_UNROLL
        for (int c = 1; c < SD; c++) s += K[t * SD + c] * den[r * SD + c];
        acc[r * TD + t] += s;
      }
  }
}

// Run-time dispatch to a functor templated on the kernel id.
#define FMMG_DISPATCH_KT(kt, KTV, ...)                                  \
  switch (kt) {                                                         \
    case LAP_S_U: { constexpr int KTV = LAP_S_U; __VA_ARGS__; } break;  \
    case LAP_D_U: { constexpr int KTV = LAP_D_U; __VA_ARGS__; } break;  \
    case STK_F_U: { constexpr int KTV = STK_F_U; __VA_ARGS__; } break;  \
    case STK_S_U: { constexpr int KTV = STK_S_U; __VA_ARGS__; } break;  \
    case STK_S_P: { constexpr int KTV = STK_S_P; __VA_ARGS__; } break;  \
    case STK_D_U: { constexpr int KTV = STK_D_U; __VA_ARGS__; } break;  \
    case STK_D_P: { constexpr int KTV = STK_D_P; __VA_ARGS__; } break;  \
    case NAV_S_U: { constexpr int KTV = NAV_S_U; __VA_ARGS__; } break;  \
    case NAV_D_U: { constexpr int KTV = NAV_D_U; __VA_ARGS__; } break;  \
    default: break;                                                     \
  }

}  // namespace fmmg
