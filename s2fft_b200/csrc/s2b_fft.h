// Ring-FFT descriptors and the parameter blocks of the element-wise kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <type_traits>

namespace s2b {

// One transform length. Tables live in pooled device arrays (FFTTables).
struct FFTDesc {
  int n;          // transform length
  int M;          // power-of-two working length (n itself, or >= 2n-1 for Bluestein)
  int logM;
  int bluestein;  // 0: n == M (radix-2 only)
  long tw_off;    // offset of exp(-2 pi i k / M), k < M/2
  long chirp_off; // Bluestein: exp(-i pi k^2 / n), k < n
  long bf_off;    // Bluestein: FFT_M(conj chirp, wrapped) / M, bit-reversed order
  // register engine (s2b_fft_reg.h; M = 2^10 .. 2^13, else -1): the twiddles of every pass in
  // the order its threads read them, and the Bluestein filter at [a T + j] for the position
  // 16 j + a that thread j holds in register a (T = M / 16)
  long rtw_off;
  long rbf_off;
};

template <typename Real>
struct FFTTables {
  using R2 = std::conditional_t<sizeof(Real) == 4, float2, double2>;
  const R2* tw;
  const R2* chirp;
  const R2* bfilt;
  const R2* rtw = nullptr;   // register-engine twiddles (FFTDesc::rtw_off)
  const R2* rbf = nullptr;   // register-engine Bluestein filters (FFTDesc::rbf_off)
};

enum RowsMode { FWD_TO_SPECTRA = 0, FWD_TO_COLS = 1, FWD_TO_RAW = 2 };

template <typename Real>
struct RowsParams {
  int L;
  int nrows;            // rows (rings) of the spectrum arrays
  int ncol;             // inverse: columns of ftm
  int mo;               // column offset (1 for mwss / healpix)
  int reality;          // inverse: fill m < 0 by conjugate symmetry
  int rings_real_2L;    // inverse, reality: mirror only on rings of 2L pixels (healpix_ifft)
  int real_out;         // inverse: write the real part only
  int real_in;          // forward: real input map
  int dual, nhalf;      // forward spectra layout
  int TR, Gs;           // forward spectra: table rows (m + kPadLo) and row stride
  int mode;             // RowsMode
  int M, m0;            // FWD_TO_RAW: out [B][nrows][M] holds X_m for m = m0 .. m0+M-1
  double scale;
  const FFTDesc* desc;  // transform descriptors
  const int* ring_desc; // per ring index into desc (nullptr: desc[0] for all)
  const long* ring_off; // element offset of ring t inside one map
  long out_batch_stride;// elements per map of the pixel-space array (f)
  const double* weights;// forward: quadrature weight per ring; inverse: output factor per ring
                        // (nullptr: 1)
  const double* phi0;   // HEALPix ring phase (nullptr: none)
  const int* col_of_ring; // forward spectra: column of ring t (nullptr: t)
  int alias_off;        // inverse, shared-memory passes: offset (complex elements) of the
                        // aliased-sum buffer in shared memory (0: none; set by the launcher)
  FFTTables<Real> tb;
  const void* in;
  void* out;
  void* zero;           // forward: a buffer the CTAs clear beside the transforms (nullptr: none)
  long zero16;          // its size in 16-byte units
};

// MW / MWSS forward resampling chain, one CTA per (m column, map).
template <typename Real>
struct ColsParams {
  int L, spin, mw;      // mw = 1: input has L MW rings, else L+1 MWSS rings
  int nin;              // rings of the input columns
  int dual, nhalf;
  int TR, Gs;           // spectra table rows and row stride
  int raw, M, m0;       // raw = 1: out [B][2L+1][M] unweighted, m = m0 .. m0+M-1
  double scale;         // overall factor of the chain
  const FFTDesc* d1;    // theta DFT over the periodic extension (2L-1 or 2L)
  const FFTDesc* d2;    // inverse DFT of length 4L
  int d2_pow2;          // 4L is a power of two (d2 without Bluestein)
  const double* weights;// 2L+1 MWSS(2L) transform weights
  const void* ph;       // [4L] complex factor of theta-DFT bin p (at p mod 4L), 0 outside
  const void* ph_adj;   // [4L] adjoint chain: conj(half-sample phase) / n1 (at p mod 4L)
  // MW: [2L+1] complex c_k, added as x_pole * c_k to the inverse-DFT output of columns with
  // odd m + s (x_pole = the input column's value on the ring theta = pi); nullptr: none
  const void* pole;
  // the chain's response (before scale and weights) to a unit impulse on the samples that are
  // their own mirror in the theta extension, for columns with odd m + s: MW [2L+1] (the pole
  // ring t = L-1, pole correction included), MWSS [2][2L+1] (t = 0, t = L; Nyquist split
  // included). Set: the register engine transforms two columns per CTA
  // (mw_cols_pair_kernel); nullptr: one column per CTA
  const void* imp;
  // MWSS real maps: the theta-Nyquist bin N (p = -L) counts half at -L and half at +L, i.e.
  // i N sin(pi k / 2) is added to the output on ring k
  int nyq_split;
  FFTTables<Real> tb;
  const void* in;       // Fc [B][ncm][nin]
  void* out;            // G  [B][half][m + kPadLo][Gs]; MWSS(2L) ring t -> row t-1,
                        // north pole -> row 2L-1, south pole -> row 2L
  // equator-symmetric output (spin 0): when set, the recursed rings go to out2 as ring
  // pairs q = 0..L-1 (rings t = q+1 and 2L-1-q) with (E, O) = G(t) +- G(2L-t) (the equator
  // q = L-1: (G, 0)), [B][half][m + kPadLo][Gs2][2], and only the pole rows to out
  void* out2;
  int Gs2;
};

}  // namespace s2b

namespace s2b {
// Ring-pair fold of the forward spectra for the equator-symmetric forward (spin 0):
// G [B][half][m + kPadLo][Gs] over nrows rings in theta order (ring t and nrows-1-t mirror
// each other) -> G2 [B][half][m + kPadLo][Gs2][2] with (E, O) = G(q) +- G(nrows-1-q) for
// q < npair = ceil(nrows / 2) (the middle ring of an odd count: (G, 0)); zero elsewhere.
// Cross mode (spin != 0, two halves, one Real2 per spectrum): G2 [B][half][m + kPadLo][Gs2][2]
// of Real4 {G_h(q), +-G_{1-h}(nrows-1-q)}, + for the first entry (l + m even), - for the
// second; the middle ring's second component is 0 (the other half counts it itself).
struct FoldParams {
  int L, nhalf, dual, TR, Gs, Gs2, nrows, npair, batch;
  int cross;
  const void* G;
  void* G2;
};
cudaError_t launch_fold_pairs(bool fp64, const FoldParams& p, cudaStream_t s);

template <typename Real>
cudaError_t launch_inv_rows(const RowsParams<Real>& p, int nrings, int batch, int maxM,
                            cudaStream_t s);
template <typename Real>
cudaError_t launch_fwd_rows(const RowsParams<Real>& p, int nrings, int batch, int maxM,
                            cudaStream_t s);
template <typename Real>
cudaError_t launch_mw_cols(const ColsParams<Real>& p, int ncm, int batch, int M1, int M2,
                           cudaStream_t s);
// Adjoint of the column chain: in = [B][2L+1][2L-1] values on the MWSS(2L) rings (row t-1 for
// ring t = 1..2L-1, north pole row 2L-1, south pole row 2L; column L-1+m), out = the
// transposed column spectra [B][nin][ncol_out] (column L-1+m+mo_out) that inv_rows reads.
template <typename Real>
cudaError_t launch_mw_cols_adj(const ColsParams<Real>& p, int ncm, int batch, int M1, int M2,
                               int ncol_out, int mo_out, cudaStream_t s);
}  // namespace s2b
