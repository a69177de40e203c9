// Summation-by-parts first-derivative and dissipation coefficients for
// sbporder 2, 3 and 4, as constant-memory tables.
//
// Row 0 is the interior stencil (2*sbporder-1 taps, centred); rows 1..
// 2*(sbporder-1) are the boundary closure rows, 3*(sbporder-1) taps each,
// applied from the block edge.  The numbers are the ones the reference
// solver uses (src/fd.cpp:53-120: rational interior/boundary weights for
// orders 2 and 3, the tabulated order-4 closure with its dissipation
// operator, and the boundary norm weight h0); they define the discrete
// operator, so any other value would be a different scheme.  Every
// translation unit that includes this header gets its own statically
// initialised copy; no run-time upload is needed.
#pragma once

#define FDF_SBP_ROWS 7
#define FDF_SBP_TAPS 9

#define FDF_SBP_TABLE(T)                                                                                   \
    {                                                                                                      \
        {/* order 2 */                                                                                     \
         {T(-0.5), T(0.), T(0.5)},                                                                         \
         {T(-1.), T(1.), T(0.)},                                                                           \
         {T(-0.5), T(0.), T(0.5)}},                                                                        \
        {/* order 3 */                                                                                     \
         {T(1. / 12.), T(-2. / 3.), T(0.), T(2. / 3.), T(-1. / 12.)},                                      \
         {T(-24. / 17.), T(59. / 34.), T(-4. / 17.), T(-3. / 34.), T(0.), T(0.)},                          \
         {T(-0.5), T(0.), T(0.5), T(0.), T(0.), T(0.)},                                                    \
         {T(4. / 43.), T(-59. / 86.), T(0.), T(59. / 86.), T(-4. / 43.), T(0.)},                           \
         {T(3. / 98.), T(0.), T(-59. / 98.), T(0.), T(32. / 49.), T(-4. / 49.)}},                          \
        {/* order 4 */                                                                                     \
         {T(-1. / 60.), T(3. / 20.), T(-3. / 4.), T(0.), T(3. / 4.), T(-3. / 20.), T(1. / 60.)},           \
         {T(-1.582533518939116), T(2.033378678700676), T(-0.141512858744873), T(-0.450398306578272),       \
          T(0.104488069284042), T(0.036577936277544), T(0.), T(0.), T(0.)},                                \
         {T(-0.462059195631158), T(0.), T(0.287258622978251), T(0.258816087376832), T(-0.069112065532624), \
          T(-0.014903449191300), T(0.), T(0.), T(0.)},                                                     \
         {T(0.071247104721830), T(-0.636451095137907), T(0.), T(0.606235523609147), T(-0.022902190275815), \
          T(-0.018129342917256), T(0.), T(0.), T(0.)},                                                     \
         {T(0.114713313798970), T(-0.290087484386815), T(-0.306681191361148), T(0.), T(0.520262285050482), \
          T(-0.051642265516119), T(0.013435342414630), T(0.), T(0.)},                                      \
         {T(-0.036210680656541), T(0.105400944933782), T(0.015764336127392), T(-0.707905442575989), T(0.), \
          T(0.769199413962647), T(-0.164529643265203), T(0.018281071473911), T(0.)},                       \
         {T(-0.011398193015050), T(0.020437334208704), T(0.011220896474665), T(0.063183694641876),         \
          T(-0.691649024426814), T(0.), T(0.739709139060752), T(-0.147941827812150), T(0.016437980868017)}}  \
    }

#define FDF_DISS_TABLE(T)                                                                                  \
    {                                                                                                      \
        {/* order 2 */                                                                                     \
         {T(0.5), T(-1.), T(0.5)},                                                                         \
         {T(-1.), T(1.), T(0.)},                                                                           \
         {T(0.5), T(-1.), T(0.5)}},                                                                        \
        {/* order 3 */                                                                                     \
         {T(-1. / 12.), T(1. / 3.), T(-1. / 2.), T(1. / 3.), T(-1. / 12.)},                                \
         {T(-8. / 17.), T(16. / 17.), T(-8. / 17.), T(0.), T(0.), T(0.)},                                  \
         {T(16. / 59.), T(-36. / 59.), T(24. / 59.), T(-4. / 59.), T(0.), T(0.)},                          \
         {T(-8. / 43.), T(24. / 43.), T(-28. / 43.), T(16. / 43.), T(-4. / 43), T(0.)},                    \
         {T(0.), T(-4. / 49.), T(16. / 49.), T(-24. / 49.), T(16. / 49.), T(-4. / 49.)}},                  \
        {/* order 4 */                                                                                     \
         {T(1. / 60.), T(-1. / 10.), T(1. / 4.), T(-1. / 3.), T(1. / 4.), T(-1. / 10.), T(1. / 60.)},      \
         {T(-0.105502234595941), T(0.316506703787823), T(-0.316506703787823), T(0.105502234595941), T(0.), \
          T(0.), T(0.), T(0.), T(0.)},                                                                     \
         {T(0.071922084408557), T(-0.227753267293765), T(0.251727295429951), T(-0.107883126612836),        \
          T(0.011987014068093), T(0.), T(0.), T(0.), T(0.)},                                               \
         {T(-0.159350793065290), T(0.557727775728513), T(-0.743637034304685), T(0.478052379195869),        \
          T(-0.159350793065290), T(0.026558465510882), T(0.), T(0.), T(0.)},                               \
         {T(0.026870684829259), T(-0.120918081731666), T(0.241836163463333), T(-0.282142190707221),        \
          T(0.201530136219444), T(-0.080612054487778), T(0.013435342414630), T(0.), T(0.)},                \
         {T(0.), T(0.018281071473911), T(-0.109686428843468), T(0.274216072108671), T(-0.365621429478228), \
          T(0.274216072108671), T(-0.109686428843468), T(0.018281071473911), T(0.)},                       \
         {T(0.), T(0.), T(0.016437980868017), T(-0.098627885208100), T(0.246569713020251),                 \
          T(-0.328759617360334), T(0.246569713020251), T(-0.098627885208100), T(0.016437980868017)}}       \
    }

static __constant__ double c_sbp_d[3][FDF_SBP_ROWS][FDF_SBP_TAPS] = FDF_SBP_TABLE(double);
static __constant__ double c_diss_d[3][FDF_SBP_ROWS][FDF_SBP_TAPS] = FDF_DISS_TABLE(double);
static __constant__ float c_sbp_f[3][FDF_SBP_ROWS][FDF_SBP_TAPS] = FDF_SBP_TABLE(float);
static __constant__ float c_diss_f[3][FDF_SBP_ROWS][FDF_SBP_TAPS] = FDF_DISS_TABLE(float);

// boundary norm weight h0 per order (fd.cpp:65, 86, 120)
static inline double fdf_sbp_h0(int order) {
    return order == 2 ? 0.5 : (order == 3 ? 17. / 48. : 13649. / 43200.);
}

template <typename T>
__device__ __forceinline__ T sbp_coef(int ord, int row, int tap);
template <>
__device__ __forceinline__ double sbp_coef<double>(int ord, int row, int tap) {
    return c_sbp_d[ord - 2][row][tap];
}
template <>
__device__ __forceinline__ float sbp_coef<float>(int ord, int row, int tap) {
    return c_sbp_f[ord - 2][row][tap];
}
template <typename T>
__device__ __forceinline__ T diss_coef(int ord, int row, int tap);
template <>
__device__ __forceinline__ double diss_coef<double>(int ord, int row, int tap) {
    return c_diss_d[ord - 2][row][tap];
}
template <>
__device__ __forceinline__ float diss_coef<float>(int ord, int row, int tap) {
    return c_diss_f[ord - 2][row][tap];
}
