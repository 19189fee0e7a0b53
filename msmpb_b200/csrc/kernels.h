// Host-side launchers of the MSM kernels. Each launcher enqueues work on the
// given stream and never synchronises; all pointers are device pointers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device.cuh"
#include "launch.cuh"

namespace msm {

constexpr int kMaxNeighbourOffsets = 4096;

// Box geometry and binning parameters (FP64)
struct Geometry {
  double A[9], Ai[9];  // row-major; columns of A are the box edge vectors
  int nc[3];           // pair cells per axis
  int M1[3];           // finest grid dims
};

// One neighbour-cell instance of the pair sweep: cell offset and the
// Cartesian offset of its origin relative to the home cell's origin
// (this includes the periodic image shift).
template <typename T>
struct CellOffset {
  int d[3];
  int pad;
  T shift[3];
  T pad2;
  double shift64[3];  // the same offset in FP64 (close pairs)
  double pad3;
};

// Short-range kernel constants. Pairs closer than sqrt(close2) are summed
// in FP64 from FP64 cell-relative positions in the mixed form: their
// forces are the largest and most sensitive to position rounding.
template <typename T>
struct PairConsts {
  T a02, inv_a02, inv_a0, two_inv_a03;
  T tau[16];
  T close2;
  double a02d, inv_a02d, inv_a0d, two_inv_a03d;
  double taud[16];
  int nu;  // MSM: the B-spline order; 0: the PME kernel erfc(beta r)/r
  // PME: beta, beta^2, 2 beta / sqrt(pi)
  T beta, beta2, c_exp;
  double betad, beta2d, c_expd;
};

// B-spline piece coefficients for the device
template <typename T>
struct SplineConsts {
  T Q[5 * 10];
  int nu;
};

// ---- atoms: binning and sorting (k_atoms.cu) ----
// prel64 (may be null): FP64 position relative to the pair-cell origin, q
template <typename T>
void launch_prep(cudaStream_t s, int N, const double *pos, const double *q,
                 const Geometry &g, int *pcell, int *gcell, int *pcount,
                 int *gcount, V4<T> *prel, V4<T> *gfrac, V4<double> *prel64,
                 int *err, double *qparts);
// blocks of launch_prep: it writes one (sum q, sum q^2) pair per block to
// qparts, which launch_qstats_final reduces
int prep_blocks(int N);
// exclusive scan of n ints into out[0..n] (out[n] = total)
size_t scan_temp_ints(int n);
void launch_scan(cudaStream_t s, const int *in, int *out, int n, int *tmp);
int scan_launches(int n);  // kernels one launch_scan of n entries issues
// two independent scans in the same launches (in0 -> out0, in1 -> out1);
// tmp: scan_temp_ints(n0) + scan_temp_ints(n1) ints
void launch_scan2(cudaStream_t s, const int *in0, int *out0, int n0, const int *in1, int *out1,
                  int n1, int *tmp);
int scan2_launches(int n0, int n1);
// Binning after the scans, one launch each: both cell scatters (pair cells,
// grid cells; with ncol > 0 also each pair-cell column's cluster count,
// ceil(atoms / 8), into clcount); both per-cell sorts (pair cells by key[atom].z, ties by atom
// index; grid cells by atom index); both gathers into sorted order, plus the
// FP64 copy of the pair records (src64/dst64, may be null).
void launch_bin_scatter(cudaStream_t s, int N, const int *pcell, const int *pstart,
                        int *pcursor, int *pperm, const int *gcell, const int *gstart,
                        int *gcursor, int *gperm, int ncol, int nc2, int *clcount);
template <typename T>
void launch_bin_sort(cudaStream_t s, int ncp, const int *pstart, int *pperm, const V4<T> *key,
                     int ncg, const int *gstart, int *gperm);
// dst[k] = src[perm[k]], cell_sorted[k] = cell[perm[k]], inv[perm[k]] = k
template <typename T>
struct GatherSide {
  const int *perm;
  const V4<T> *src;
  const int *cell;
  V4<T> *dst;
  int *cell_sorted, *inv;
};
template <typename T>
void launch_bin_gather(cudaStream_t s, int N, const GatherSide<T> &p,
                       const V4<double> *src64, V4<double> *dst64, const GatherSide<T> &g);
struct CombineArgs {
  int N;
  double w0, coeff1, coeff2, gamma0_over_a0;
  const double *q;
  const double *qstats;  // [qsum, q2sum] after the final reduction
  int nqparts;
  const double *qparts;
  double *force;     // N*3 or NULL
  double *phi;       // N or NULL
  double *epart;     // per-block partial sums of w0 * q_i * phi_short_i / 2
};
template <typename T>
void launch_combine(cudaStream_t s, const CombineArgs &a, const int *pinv,
                    const int *ginv, const V4<T> *pout, const V4<T> *gout,
                    int nblocks);
int combine_blocks(int N);
struct EnergyArgs {
  const double *qparts;  // nqparts x 2
  int nqparts;
  const double *short_parts;
  int nshort;
  const double *grid_parts;
  int ngrid;
  double w0, coeff1, coeff2, gamma0_over_a0;
  double *energy;  // device scalar
  double *qstats;  // device [qsum, q2sum]
  double grid_scale = 1.0;  // factor on the grid energy q^1 . e^1 / 2
};
void launch_energy_total(cudaStream_t s, const EnergyArgs &a);
void launch_qstats_final(cudaStream_t s, const double *qparts, int nqparts,
                         double *qstats);

// ---- short-range pair sum (k_pair.cu) ----
// pos64_sorted: FP64 cell-relative positions in the same order (used for
// close pairs in the mixed form; may be null for T = double)
template <typename T>
void launch_pair(cudaStream_t s, int N, const V4<T> *pos_sorted,
                 const V4<double> *pos64_sorted, const int *cell_sorted,
                 const int *cell_start, const Geometry &g,
                 const CellOffset<T> *offsets, int noff,
                 const PairConsts<T> &pc, V4<T> *out);

// cluster form (k_pair_clusters.cu): clusters of 8 z-ordered atoms per
// pair-cell column, one warp per i-cluster, 8 x 4 pair tiles
constexpr int kMaxColumnOffsets = 1024;
// A neighbour column (du, dv) and the Cartesian offset of its origin,
// A (du/nc0, dv/nc1, 0), periodic image included.
struct ColumnOffset {
  int du, dv, pad[2];
  double base[3];
  double pad2;
};
struct ClusterInfo {
  int first;     // sorted index of the first atom
  int n;         // atoms (1..8)
  int col;       // column cx * nc1 + cy
  int czf, czl;  // cell z of the first and the last atom
  int pad[3];
  float4 c, h;   // bounding box centre and half extents (cluster frame)
};
struct UnitBox {  // half cluster; c.w holds the cluster's czf (int bits)
  float4 c, h;
};
template <typename T>
struct PairClusterArgs {
  int maxcl, ncol, nc0, nc1, nc2, K2, ncoloff;
  float rbox2;      // squared cutoff plus margin for the box test
  float rnear2;     // squared close-pair distance plus margin (FP32 form:
                    // j atoms this near the i-cluster box take the checked path)
  int ortho;        // orthorhombic box: per-column z windows from the xy gap
  int ozero;        // index of the (0, 0) column offset
  float cw[3];      // cell widths along x, y, z (orthorhombic boxes)
  double cz[3];     // A (0, 0, 1/nc2): one cell along the column
  const int *start;     // pair-cell starts (ncell + 1)
  const int *clstart;   // first cluster of each column (ncol + 1)
  const ColumnOffset *coloff;
  const ClusterInfo *info;
  const UnitBox *ubox;
  const V4<T> *cpos;          // maxcl x 8 (cluster frame, charge in w)
  const V4<double> *cpos64;   // FP64 copy (mixed form) or null
  V4<T> *out;                 // per sorted atom: force / q_i and potential
  int *err;
  int self_images;            // a lattice vector shorter than a0: an atom's
                              // own images reach its tiles and are skipped
  // unit lists (the adjoint's cluster pass, mixed form): per i-cluster a
  // region of lcap entries {unit, item code | first cell | atom mask} of the
  // half-cluster units that pass the box test, far ones from the front, near
  // ones (within the close distance of the box, or of the cluster itself)
  // from the back; lcnt = {far, near} counts, which may exceed lcap (the
  // pass then sweeps that cluster's candidates itself). Null: no lists.
  int2 *list;
  int2 *lcnt;
  int lcap;
};
int cluster_capacity(int N, int ncol);
// entries per i-cluster of the unit lists
constexpr int kUnitListCap = 512;
// builds the unit lists of a.list / a.lcnt (one warp per i-cluster, few
// registers; FP32 boxes in both precisions)
template <typename T>
void launch_pair_list(cudaStream_t s, const PairClusterArgs<T> &a);
// src64: FP64 cell-relative positions and charges in sorted order
template <typename T>
void launch_cluster_fill(cudaStream_t s, int maxcl, int ncol, int nc2,
                         const int *start, const int *clstart, const int *pcs,
                         const V4<double> *src64, const double cz[3], V4<T> *cpos,
                         V4<double> *cpos64, ClusterInfo *info, UnitBox *ubox);
template <typename T>
void launch_pair_clusters(cudaStream_t s, const PairClusterArgs<T> &a,
                          const PairConsts<T> &pc);
// adjoint short-range pass on the cluster sweep (mixed form; the FP64 form
// uses launch_adj_pair): fbs = Fbar in pair-cell order, fslot scratch of
// maxcl x 8 records (Fbar gathered into cluster-slot order), out_a = (E, psi),
// out_b = (h, 0) per sorted atom, as launch_adj_pair
template <typename T>
bool adj_pair_clusters_supported();
template <typename T>
void launch_adj_pair_clusters(cudaStream_t s, const PairClusterArgs<T> &a,
                              const PairConsts<T> &pc, const V4<T> *fbs, V4<T> *fslot,
                              V4<T> *out_a, V4<T> *out_b);

// ---- grid transfers (k_grid.cu) ----
// variant 0: tile scatter with a fold (scratch: anterp_scratch_elems
// values; grids smaller than nu along an axis use the slab gather);
// otherwise the slab-staged gather
size_t anterp_scratch_elems(const int M[3], int nu);
bool anterp_tiles_supported(const int M[3], int nu);
// per-axis cover table of the fold (5 ints per grid index and axis)
std::vector<int> anterp_fold_table(const int M[3], int nu);
template <typename T>
void launch_anterpolate(cudaStream_t s, const int M[3], const V4<T> *atoms,
                        const int *cell_sorted, const int *cell_start,
                        const SplineConsts<T> &sc, T *grid, int variant, int *err,
                        long natoms, T *scratch, const int *fold_tab);
template <typename T>
void anterpolate_prepare();
template <typename T>
void launch_interpolate(cudaStream_t s, int N, const int M[3],
                        const V4<T> *atoms, const int *cell_sorted,
                        const T *grid, const SplineConsts<T> &sc,
                        const Geometry &g, V4<T> *out);
template <typename T>
void launch_restrict(cudaStream_t s, const int Mf[3], const T *fine,
                     T *coarse, const double *J, int nu);
template <typename T>
void launch_prolong_add(cudaStream_t s, const int Mf[3], const T *coarse,
                        T *fine, const double *J, int nu);
template <typename T>
void launch_grid_dot(cudaStream_t s, size_t n, const T *a, const T *b,
                     double *partials, int nparts);
int grid_dot_blocks(size_t n);

// ---- per-level direct stencil (k_stencil.cu) ----
struct StencilShape {
  int M[3];   // grid dims
  int S[3];   // stencil dims
  int P[3];   // padded input dims (P[2] rounded up for 16-byte rows)
  int sym;    // 1: taps mirror-symmetric in x and y, S0 and S1 odd (folded
              // sweep, taps given as the folded (S0/2+1) x (S1/2+1) rows)
  int store;  // 1: e = w K q (overwrite); 0: e += w K q
};
// CTA tile of the stencil sweep: nz x ty threads, each with tx x R outputs
struct StencilTile {
  int nz = 0, ty = 0, tx = 0;
  int nsplit = 1;  // CTAs sharing one output tile, each over a run of tap planes
  int r = 0;       // z outputs per thread of the folded sweep (0: the default)
};
// z outputs per thread of a tile (the precision's default unless the tile
// picks the folded sweep's alternative)
int stencil_tile_r(const StencilTile &tile, bool fp64);
// alternative z outputs per thread of the folded sweep for this shape, or 0
int stencil_alt_r(const StencilShape &sh, bool fp64);
StencilTile stencil_default_tile(const StencilShape &sh, bool fp64);
bool stencil_templated(const StencilShape &sh);
// row pitch of the tap array: S2 rounded up to 16 bytes (rows zero padded)
int stencil_tap_pitch(int S2, bool fp64);
// folded taps for a symmetric stencil: kf[i][j][k], i <= S0/2, j <= S1/2,
// the mean of the (up to four) mirror images kh[S0/2 +- i][S1/2 +- j][k],
// rows padded to the tap pitch. Returns false (and leaves kf empty) when
// kh is not mirror-symmetric in x and y to 1e-12 of its largest tap or
// S0, S1 are even.
bool stencil_fold_taps(const double *kh, const int S[3], bool fp64,
                       std::vector<double> &kf);
// padded input dims that keep every tile load of `tile` inside the buffer
void stencil_padded_dims(const StencilShape &sh, const StencilTile &tile,
                         bool fp64, int P[3]);
// one-time kernel attributes (dynamic shared memory); <0 if unsupported
template <typename T>
int stencil_prepare(const StencilShape &sh, const StencilTile &tile);
template <typename T>
void launch_pad(cudaStream_t s, const StencilShape &sh, const T *q, T *padded);
// tile autotuner (tune.cu)
bool stencil_tuning_enabled();
std::vector<StencilTile> stencil_candidates(const StencilShape &sh, bool fp64);
template <typename T>
StencilTile stencil_autotune(cudaStream_t s, int device, const StencilShape &sh,
                             const StencilTile &fallback, const T *padded,
                             size_t padded_cap, const T *kh, int khz, T *e,
                             T *part, size_t part_cap, double *best_ms);
// kh: S0 x S1 x khz taps (z fastest); part: tile.nsplit x M0*M1*M2
// scratch for split tap sums (unused when nsplit == 1)
template <typename T>
void launch_stencil(cudaStream_t s, const StencilShape &sh,
                    const StencilTile &tile, const T *padded, const T *kh,
                    int khz, T weight, T *e, T *part);
int stencil_launches(const StencilShape &sh, const StencilTile &tile);

// ---- adjoint (k_adjoint.cu, k_grid.cu) ----
struct AdjointCombineArgs {
  int N;
  double w0, coeff1, coeff2, gamma0_over_a0;
  const double *q;       // input order
  const double *qstats;  // [qsum, q2sum]
  const double *fbar;    // force cotangent, N*3, input order
  double ubar;           // energy cotangent
  double *dq;            // N or null
  double *dr;            // N*3 or null
};
template <typename T>
void launch_adj_gather(cudaStream_t s, int N, const int *perm, const double *fbar, V4<T> *out);
template <typename T>
void launch_adj_dipoles(cudaStream_t s, int N, const int *perm, const double *q,
                        const double *fbar, const Geometry &g, V4<T> *out);
template <typename T>
void launch_adj_pair(cudaStream_t s, int N, const V4<T> *ps, const V4<T> *fbs, const int *pcs,
                     const int *start, const Geometry &g, const CellOffset<T> *off, int noff,
                     const PairConsts<T> &pc, V4<T> *out_a, V4<T> *out_b);
template <typename T>
void launch_adj_combine(cudaStream_t s, const AdjointCombineArgs &a, const int *pinv,
                        const int *ginv, const V4<T> *pout, const V4<T> *gout,
                        const V4<T> *adj_a, const V4<T> *adj_b, const V4<T> *adj_g,
                        const V4<T> *adj_h);
// dipole anterpolation (tile scatter; grids >= nu per axis) and the adjoint
// interpolation (value and gradient of ed, Hessian of e1 times Fbar)
template <typename T>
void launch_adj_anterpolate(cudaStream_t s, const int M[3], const V4<T> *atoms,
                            const int *cell_sorted, const int *cell_start,
                            const SplineConsts<T> &sc, const V4<T> *dip, T *grid,
                            T *scratch, const int *fold_tab);
template <typename T>
void launch_adj_interpolate(cudaStream_t s, int N, const int M[3], const V4<T> *atoms,
                            const int *cell_sorted, const int *gperm, const double *fbar,
                            const T *ed, const T *e1, const SplineConsts<T> &sc,
                            const Geometry &g, V4<T> *out_g, V4<T> *out_h);

// ---- level stencils on the device for a new box (k_setup.cu) ----
struct LevelStencilArgs {
  double A[9];      // row-major; columns are the box edge vectors
  double as[3];     // column norms of A^-1
  double al;        // cutoff of the level, a_l
  double tau[16];   // softening polynomial coefficients
  int nu;
  int g[3];         // level grid dims
  int sd[3];        // stencil dims
  int oms;          // row stride of the omega' table (x, y, z rows)
};
// kp: sd0 x sd1 rows of the tap pitch; kf (may be null): folded rows;
// om: omega'_x, omega'_y, omega'_z rows of a.oms; work: 3 sd^3 doubles
template <typename T>
void launch_level_stencil(cudaStream_t s, const LevelStencilArgs &a, const double *om,
                          double *work, T *kp, T *kf, bool fp64);

// ---- top-level FFT solve (k_fft.cu) ----
bool top_solve_supported(const int M[3]);
int top_solve_launches(const int M[3]);  // kernels one launch_top_solve issues
void top_solve_prepare();
template <typename T>
void launch_top_solve(cudaStream_t s, const int M[3], const T *q,
                      const double *khat, double weight, double2 *buf0,
                      double2 *buf1, T *e);

}  // namespace msm
