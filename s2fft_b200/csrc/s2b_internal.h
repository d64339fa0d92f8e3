// Internal declarations shared by the host plan code and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace s2b {

// Renormalisation constants of the scaled recursion state.
// A state stores a mantissa v and an integer exponent e; its true value is
// v * 2^(kScale * e). e < 0 means "below significance": the state is advanced
// but contributes nothing to the projection. Every kRenorm steps a state with
// |v| > 2^kThresh is rescaled by 2^-kScale (e += 1).
template <typename Real>
struct Scaling;
template <>
struct Scaling<float> {
  static constexpr double kThresh = 48.0;  // log2 of the rescale trigger
  static constexpr double kScale = 112.0;  // log2 of one exponent unit
  static constexpr double kSignif = -60.0; // log2 of the significance floor
  static constexpr float kTrig = 281474976710656.0f;          // 2^48
  static constexpr float kDown = 1.9259299443872359e-34f;    // 2^-112
};
template <>
struct Scaling<double> {
  static constexpr double kThresh = 400.0;
  static constexpr double kScale = 800.0;
  static constexpr double kSignif = -200.0;
  static constexpr double kTrig = 0x1p400;
  static constexpr double kDown = 0x1p-800;
};

// Coefficient tables indexed by m are stored with kPadLo zero rows on both
// sides of 0 <= m < L (row = m + kPadLo), so that every R-step group of the
// latitudinal kernel is one fixed-size contiguous copy.
constexpr int kPadLo = 8;
__host__ __device__ inline int tab_rows(int L) { return L + 2 * kPadLo; }
__host__ __device__ inline int round4(int x) { return (x + 3) & ~3; }

// One recursed ring (pole rings are handled separately, in closed form).
struct RingInfo {
  double B;    // 2 cot(theta)
  double A;    // 2 / sin(theta)
  double lc;   // log2 cos(theta/2)
  double ls;   // log2 sin(theta/2)
};

// Latitudinal (Wigner-d recursion + projection) launch parameters.
struct LatParams {
  int L, L0, spin;
  int nrings;       // recursed rings
  int nclass;       // C: l classes (CTAs along l); l = j + C*(ql + QA*k)
  int Qp;           // l slots per class (padded to a multiple of 4)
  int nhalf;        // recursion halves handled by this launch (1 or 2)
  int batch;
  const RingInfo* rings;
  const int* ring_row;   // row of ring r in the ftm array (inverse out / forward in)
  const void* seeds;     // [nhalf][C][Qp][nrings] {mantissa, exponent}
  const void* H;         // [C][tab_rows][Qp] monic recursion coefficient h_{l,m}
  // inverse: in = F  [batch][nhalf][C][tab_rows][Qp] Real2 (Real4 when dual)
  //          out = ftm [batch][nrows][ncol] Real2 (accumulated with atomics)
  // forward: in = G  [batch][nhalf][tab_rows][Gs] Real2 (Real4 when dual);
  //          ring r of the launch is row r of G (pole rows, if any, come after)
  //          out = acc [batch][nhalf][C][L (m)][Qp] Real2 (accumulated with atomics)
  int Gs;           // forward: row stride of G (multiple of 4)
  const void* lam;  // [nhalf][tab_rows][Ls] lambda(theta_r, m) = 2 (n - m cos) / sin, rounded once
  int Ls;           // row stride of lam (multiple of 4, >= nrings)
  int* status;      // device status word: nonzero after a timed-out wait
  const void* in;
  void* out;
  int nrows;        // rows of the ftm array
  int ncol;         // inverse: columns of ftm
  int mo;           // inverse: column offset (1 for mwss / healpix)
  int reality;      // inverse: only m >= 0 is produced
};

// launchers (latitudinal.cu)
cudaError_t launch_latitudinal(bool fp64, bool forward, bool dual, const LatParams& p,
                               cudaStream_t s);
cudaError_t launch_seeds(bool fp64, int L, int L0, int spin, int nhalf, const RingInfo* rings,
                         int nrings, const double* lbin, void* seeds, cudaStream_t s);
int lat_nclass(bool fp64, int L);
cudaError_t launch_lambda(bool fp64, int L, int spin, int nhalf, const RingInfo* rings, int nrings,
                          int Ls, void* lam, cudaStream_t s);
int lat_qp(bool fp64, int L);

// Records msg as the calling thread's s2b_last_error() text and returns code.
int set_last_error(int code, const char* msg);
size_t seed_bytes(bool fp64, int L, int nhalf, int nrings);

}  // namespace s2b
