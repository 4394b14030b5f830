// Device data layout of the batched coni pipeline.
#pragma once
#include <cstdint>
#include "pfg_int.cuh"

namespace pfg {

constexpr int MH = 64;          // largest h11 (pfg_max_h11)
constexpr int MD = MH - 1;      // largest search dimension
constexpr unsigned FULL = 0xffffffffu;

// A direction gets GCD rows (pruning only) when its estimated search tree
// has at least this many nodes: below that, building the rows costs more
// device time than the nodes they could remove.
constexpr double GCD_MIN_TREE_DEFAULT = 1.0e3;

// per-direction status (device); the ABI's pstat carries the same codes
enum : int {
    ST_OK = 0,          // searched, points emitted
    ST_EMPTY = 3,       // M0 == 0 on the whole lattice and M0min > 0: no points
    ST_PENDING = 4,     // set up, not searched yet
    ST_WANT_ROWS = 5,   // (internal) set up but for its GCD rows: queued for setup phase 3
    ST_RANGE = -8,      // a coordinate range exceeds int32 (reference status -8)
    ST_NOT_PD = -9,     // ellipsoid matrix not positive definite (reference -9)
    ST_FLOAT = -11,     // FP32 error bound exceeded: search again in FP64
    ST_OVERFLOW = -20,  // exact setup values beyond the device's fixed-width integers
    ST_PRECISION = -21, // FP64 factor not certified (ill-conditioned beyond bounds)
    ST_WAIT = -22,      // a bounded device wait ran out
    ST_NONPOS = -30,    // (internal, never reported) a Gram-Schmidt norm <= 0 in an LLL
};

struct Geo {
    int h, d, use_f32;
    int coni;                   // 1: coni (M0 cut, strict GCD cut on K[1:]); 0: non-coni (none, non-strict on K)
    int64_t Q, qmax, linmin;
    int64_t koff, moff;         // offsets of kappa (h^3) and Mbasis (h^2)
    int64_t slab_len;           // int64 words of one direction's slab
};

// Per-direction metadata written by the setup kernel.
struct Dir {
    int geo, h, d, status;
    int m0_level;               // level at which M0 is determined (-1: M0 == 0)
    int pad;                    // setup step that failed (diagnostics), else 0
    int wide;                   // 1: mat has entries beyond int32 (the search reads it from the slab)
    int pad2;
    int64_t g_lin;              // M0 = g_lin * c[d-1] (cut-aware basis)
    uint64_t hrows;             // bit j: the GCD row with pivot j is kept
    int64_t slab;               // offset (int64 words) of the slab
    double slack_chol;          // certified Cholesky backward-error margin on q
};

// Slab of one direction (int64 words), dimensions h, d:
//   BT   d x h  int64   Binter^T: BT[a][r] = Binter[r][a]
//   ZT   d x h  int64   (Z Binter)^T
//   MAT  d x d  int64   ellipsoid matrix
//   H    d x d  int64   GCD rows, transposed: H[c d + j] = entry c of the row whose
//                        first nonzero is at column j
//   U64  d x d  double  upper Cholesky factor (U^T U = mat + a certified perturbation)
//   U32  d x d  float   U64 rounded to float (padded to whole words)
//   UI64 d      double  1 / U64[i][i]
//   UI32 d      float   1 / U32[i][i]
struct Slab {
    int64_t bt, zt, mat, H, u64, u32, ui64, ui32, len;
};

PFG_HD Slab slab_layout(int h, int d)
{
    Slab s;
    s.bt = 0;
    s.zt = s.bt + (int64_t)d * h;
    s.mat = s.zt + (int64_t)d * h;
    s.H = s.mat + (int64_t)d * d;               // (the search reads a wide mat as H - d d)
    s.u64 = s.H + (int64_t)d * d;
    s.u32 = s.u64 + (int64_t)d * d;
    s.ui64 = s.u32 + ((int64_t)d * d + 1) / 2;
    s.ui32 = s.ui64 + d;
    s.len = s.ui32 + (d + 1) / 2;
    return s;
}

// One point found by the search: direction, exact q, and its coordinates in
// the direction's basis (M = Binter c and Kn = Z Binter c are formed later).
struct PointHdr {
    int32_t pid;
    int32_t pad;
    int64_t q;
};

}  // namespace pfg
