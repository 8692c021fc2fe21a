// Device-resident data shared by the hot-path kernels.
//
// Field storage keeps the reference plane layout (src/auxfield.cpp:45-68,
// src/geometry.cpp:105-108): data[k*plane_size + e*np*np + i*np + j], i = s
// row, j = r column; in Fourier space plane 0 = Re mode 0, plane 1 = Nyquist,
// planes 2m / 2m+1 = Re / Im of mode m (femlib/fourier.c:56-63).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace stx {

struct DevGeom {
  int np, nel, nz, npnp, next, nint, plane_size;
  const double* D;      // [np*np] derivative matrix
  const double* Q1;     // [nel*npnp] geometric factors
  const double* Q2;
  const double* Q3;
  const double* Q4;
  const double* drdx;
  const double* drdy;
  const double* dsdx;
  const double* dsdy;
  const int* emap;      // [npnp] boundary-major traverse
  const int* pmap;      // [npnp] inverse of emap
  const int* family;    // [nel] geometry family
  // Elements grouped into chunks of one family (for the batched element
  // kernels): chunk c covers elem_sorted[chunk_start[c] .. + chunk_count[c]).
  int nchunk, chunk_max;
  const int* chunk_start;
  const int* chunk_count;
  const int* elem_sorted;
  const int4* chunk_desc;  // [nchunk] (chunk_start, chunk_count, family, 0): one load per block
  int pdl;                 // 1: the DNS step's kernels launch programmatically dependent (token STX_PDL_STEP)
};

struct DevNumbering {
  int nglobal, nsolve, nband;
  const int* btog;      // [nel*next]
  const int* bmask;     // [nel*next]
  const int* emask;     // [nel]
  const double* imass;  // [nglobal]
  int nedge;            // boundary edges with a BC
  const int* edge_gid;  // [nedge*np] global id of each edge node
  const int* edge_kind; // [nedge]  'D' or 'N'
  const double* edge_area;  // [nedge*np]
  const double* mixdiag;    // [nglobal] mixed-BC diagonal (K x side weights), or null
  int ness, nnat;           // edges of kind 'D' / 'N' (kernels with nothing to do are not launched)
};

// One tiled product y += scale A x for the planes of a Fourier mode, the
// matrix at l2_pack + moff: symmetric packed (ncol = 0, order n; x_i read
// and y_i accumulated at position idx[i] of the planes' skeleton vectors,
// x_pin taken as zero) or general n x ncol (y_i at idx[i], x_j read at
// idx_col[j]).
struct SymProblem {
  long long moff;
  int n, mode, pin;
  const int* idx;
  int ncol;
  const int* idx_col;
  double scale;
};

// The tiles one warp of a packed product streams: `count` tiles in packed
// order from tile q of problem `prob`, continuing into the following
// problems.
struct SymWarp {
  int prob, q, count;
};

// A ModalMatrixSys on the device: one MatrixSys per locally held mode.
struct DevModal {
  int nmodes, method, nfamily;
  int mode0;                      // mode of blockIdx.y = 0: a launch covers modes [mode0, mode0 + nmodes)
  int nband, ns_stride;           // band width, rows reserved per mode
  int nbp;                        // factor row stride (nband rounded up to even)
  long long mode_stride;          // doubles between modes' factors (256-byte multiple)
  long long dinv_stride;          // doubles between modes' inverse diagonal blocks
  const double* D;                // [np*np] derivative matrix of the operators: the
                                  // SVV-stabilised one for viscous systems with SVV
  const double* lambda2;          // [nmodes]
  const double* betak2;           // [nmodes]
  const int* nsolve;              // [nmodes]
  const double* hbi;              // [nmodes][nfamily][next][nint]
  const double* hii;              // [nmodes][nfamily][nint][nint]
  // Element operators of the element kernels, rows padded: recovery row i
  // (columns in natural node order) = -hbi[b][i] at boundary node b,
  // hii^-1[i][j] at interior node j; condensation row b = hbi[b][.] over the
  // interior nodes in boundary-major order.
  const double* ew;               // [nmodes][nfamily][nint][ew_ld]
  int ew_ld;
  const double* eb;               // [nmodes][nfamily][next][eb_ld]
  int eb_ld;
  const double* fwd;              // [nmodes][mode_stride]: rows of U^T, stride nbp
  const double* bwd;              // [nmodes][mode_stride]: rows of reversed U
  const double* dinv_fwd;         // [nmodes][dinv_stride]: 16x16 inverse diagonal blocks
  const double* dinv_bwd;
  int* status;                    // device status word (0 = ok)
  int sym_warps;                  // warps per block of the packed products (token STX_SYM_WARPS)
  int sym_regcap;                 // 1: their register-capped build (token STX_SYM_REGCAP)
  int elem_twoblock;              // 1: element kernels split rows to run two blocks per SM (STX_ELEM_TWOBLOCK)
  int pdl;                        // 1: the solve's kernels launch programmatically dependent (STX_PDL)
  unsigned long long wait_ns;     // bound of the element and skeleton kernels' first
                                  // wait per copy (token STX_WAIT_NS, default 2 s)
  const double* pc;               // JACPCG: [nmodes][npts]
  int npts;
  // Two-level condensation (patches + interface system, both through packed
  // symmetric inverses); l2 = 0 when the single banded factor above is used.
  int l2;
  int npatch, pfam, nI_max, nB_max, niface;
  const int* p_family;            // [npatch]
  const int* p_nI;                // [npatch]
  const int* p_nB;                // [npatch]
  const int* p_Igid;              // [npatch][nI_max] skeleton ids of interior nodes
  const int* p_Biid;              // [npatch][nB_max] interface ids of boundary nodes
  const int* skel_of;             // [niface] skeleton id of each interface unknown
  const int* pin;                 // [nmodes] pinned interface id or -1
  const double* l2_pack;          // packed symmetric inverses (symtile.hpp layout)
  const SymProblem* prob_patch;   // S_II^-1 products: one per (patch, mode)
  const SymWarp* warp_patch;
  int nwarp_patch;
  const SymProblem* prob_iface;   // interface products: one per mode
  const SymWarp* warp_iface;
  int nwarp_iface;
  const SymProblem* prob_gen;     // recovery products -G x_B: one per (patch, mode)
  const SymWarp* warp_gen;
  int nwarp_gen;
  const double* l2_sc;            // [nmodes][nfamily][next][l2_sc_ld] element Schur complements
  int l2_sc_ld;
  const int* l2_ncode;            // [nel][next], elements in chunk order: skeleton id << 2 | class
                                  // (0 essential, 1 patch-interior, 2 interface node)
  // Mixed precision (l2_pack32 set): the packed matrices of l2_pack held in
  // FP32 at the same entry offsets, and `refine` FP64 residual corrections
  // of the skeleton solution.
  const float* l2_pack32;
  int refine;
};

}  // namespace stx
