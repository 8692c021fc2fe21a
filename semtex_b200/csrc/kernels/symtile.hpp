// Packed storage of a symmetric n x n matrix for the tiled products of the
// two-level skeleton solve: the lower triangle of 32 x 32 tiles (I >= J),
// tile-row-major, the last tile row only as tall as the matrix needs
// (h = n - 32 (T - 1) rows, stored rounded up to a multiple of 4).  Diagonal
// tiles hold both triangles; columns past n are zero.  Within a tile, row r
// occupies 33 entries (entry (r, c) at r*33 + c, the 33rd zero: tile_pos),
// so that a warp reading a tile row (lanes over c) or a tile column (lanes
// over r) touches every bank once and every address is a constant offset.
// (A layout of 4 x 4 quadrants, which FP64 tensor-core fragments read
// conflict-free, was measured slower: with one or two planes per tile the
// m8n8k4 products use 2 of their 8 columns.)  Offsets and sizes count entries;
// with doubles or floats alike every tile is a multiple of 16 bytes and
// starts on a 16-byte boundary: one bulk copy each.
#pragma once

#include <cstddef>

namespace stx {

constexpr int kSymTile = 32;
constexpr int kSymLd = kSymTile;  // entries per stored tile row

// Entry (r, c) of a tile, and its inverse (c = 32: the zero padding entry).
__host__ __device__ inline int tile_pos(int r, int c) { return r * kSymLd + c; }
__host__ __device__ inline void tile_rc(int w, int& r, int& c) {
  r = w / kSymLd;
  c = w - r * kSymLd;
}

__host__ __device__ inline int sym_tiles(int n) { return (n + kSymTile - 1) / kSymTile; }

__host__ __device__ inline int sym_last_rows(int n) { return n - kSymTile * (sym_tiles(n) - 1); }

// Rows of tile row I, and rows stored for it.
__host__ __device__ inline int sym_rows(int n, int I) { return I < sym_tiles(n) - 1 ? kSymTile : sym_last_rows(n); }
__host__ __device__ inline int sym_rows_stored(int n, int I) { return (sym_rows(n, I) + 3) / 4 * 4; }

// Doubles of the packed matrix.
__host__ __device__ inline long long sym_size(int n) {
  if (n <= 0) return 0;
  const long long T = sym_tiles(n), hs = (sym_last_rows(n) + 3) / 4 * 4;
  return (T - 1) * T / 2 * kSymTile * kSymLd + T * hs * kSymLd;
}

// Doubles from the matrix start to tile (I, J), J <= I.
__host__ __device__ inline long long sym_tile_offset(int n, int I, int J) {
  const int T = sym_tiles(n);
  const long long full = static_cast<long long>(kSymTile) * kSymLd;
  if (I < T - 1) return (static_cast<long long>(I) * (I + 1) / 2 + J) * full;
  return static_cast<long long>(T - 1) * T / 2 * full + static_cast<long long>(J) * sym_rows_stored(n, I) * kSymLd;
}

// Number of tiles and the tile (I, J) at packed position q (row-major over J <= I).
__host__ __device__ inline int sym_ntiles(int n) {
  const int T = sym_tiles(n);
  return T * (T + 1) / 2;
}

__host__ __device__ inline void sym_tile_at(int q, int& I, int& J) {
  int i = 0;
  while ((i + 1) * (i + 2) / 2 <= q) ++i;
  I = i;
  J = q - i * (i + 1) / 2;
}

// Pack the symmetric matrix A (row-major, leading dimension lda) into out
// (sym_size(n) doubles, zero-initialised by the caller).
inline void sym_pack(int n, const double* A, size_t lda, double* out) {
  const int T = sym_tiles(n);
  for (int I = 0; I < T; ++I)
    for (int J = 0; J <= I; ++J) {
      double* t = out + sym_tile_offset(n, I, J);
      const int h = sym_rows(n, I);
      for (int r = 0; r < h; ++r)
        for (int c = 0; c < kSymTile; ++c) {
          const int i = kSymTile * I + r, j = kSymTile * J + c;
          t[tile_pos(r, c)] = j < n ? A[static_cast<size_t>(i) * lda + j] : 0.0;
        }
    }
}

// General (rectangular) nr x nc matrices in the same tile format: all
// T_r x T_c tiles, tile-row-major, last tile row stored as tall as needed
// (rounded up to a multiple of 4), columns past nc zero.
__host__ __device__ inline int gen_ntiles(int nr, int nc) { return sym_tiles(nr) * sym_tiles(nc); }

__host__ __device__ inline long long gen_size(int nr, int nc) {
  if (nr <= 0 || nc <= 0) return 0;
  const long long Tr = sym_tiles(nr), Tc = sym_tiles(nc), hs = (sym_last_rows(nr) + 3) / 4 * 4;
  return (Tr - 1) * Tc * kSymTile * kSymLd + Tc * hs * kSymLd;
}

__host__ __device__ inline long long gen_tile_offset(int nr, int nc, int I, int J) {
  const int Tr = sym_tiles(nr), Tc = sym_tiles(nc);
  const long long full = static_cast<long long>(kSymTile) * kSymLd;
  if (I < Tr - 1) return (static_cast<long long>(I) * Tc + J) * full;
  return static_cast<long long>(Tr - 1) * Tc * full + static_cast<long long>(J) * sym_rows_stored(nr, I) * kSymLd;
}

inline void gen_pack(int nr, int nc, const double* A, size_t lda, double* out) {
  const int Tr = sym_tiles(nr), Tc = sym_tiles(nc);
  for (int I = 0; I < Tr; ++I)
    for (int J = 0; J < Tc; ++J) {
      double* t = out + gen_tile_offset(nr, nc, I, J);
      const int h = sym_rows(nr, I);
      for (int r = 0; r < h; ++r)
        for (int c = 0; c < kSymTile; ++c) {
          const int i = kSymTile * I + r, j = kSymTile * J + c;
          t[tile_pos(r, c)] = j < nc ? A[static_cast<size_t>(i) * lda + j] : 0.0;
        }
    }
}

}  // namespace stx
