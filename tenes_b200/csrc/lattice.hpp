// Unit-cell geometry (SquareLattice, src/SquareLattice.hpp:54-163 and
// src/SquareLattice.cpp:48-137): site index <-> (x, y), neighbour tables
// (0 = left, 1 = top, 2 = right, 3 = bottom), skew boundary condition.
#pragma once

#include <array>
#include <numeric>
#include <vector>

#include "common.hpp"

namespace tg {

struct Lattice {
  int LX = 0, LY = 0, N = 0, skew = 0;
  int LX_noskew = 0, LY_noskew = 0;
  std::vector<int> pdim;                 // physical dimension per site
  std::vector<std::array<int, 4>> vdim;  // virtual dims per site
  std::vector<std::vector<int>> list;    // [x][y] -> site
  std::vector<std::array<int, 4>> nn;

  Lattice() = default;
  Lattice(int X, int Y, int skew_in) : LX(X), LY(Y), N(X * Y) {
    if (X <= 0) fail(TG_E_INPUT, "Lattice.X should be positive");
    if (Y <= 0) fail(TG_E_INPUT, "Lattice.Y should be positive");
    skew = skew_in % LX;  // C++ remainder, as the reference member init
    LX_noskew = LX;
    if (skew_in == 0) {
      LY_noskew = LY;
    } else {
      int s = ((skew_in % LX) + LX) % LX;
      if (s == 0) fail(TG_E_INPUT, "skew must not be a multiple of L_sub[0]");
      int l = LX / std::gcd(LX, s) * s;
      LY_noskew = LY * (l / s);
    }
    list.assign(LX, std::vector<int>(LY));
    for (int ix = 0; ix < LX; ++ix)
      for (int iy = 0; iy < LY; ++iy) list[ix][iy] = ix + iy * LX;
    nn.resize(N);
    for (int iy = 0; iy < LY; ++iy)
      for (int ix = 0; ix < LX; ++ix) {
        const int i = ix + iy * LX;
        nn[i][0] = list[(ix - 1 + LX) % LX][iy];
        nn[i][1] = list[ix][(iy + 1) % LY];
        nn[i][2] = list[(ix + 1) % LX][iy];
        nn[i][3] = list[ix][(iy - 1 + LY) % LY];
      }
    if (skew != 0) {
      for (int ix = 0; ix < LX; ++ix) {
        nn[ix][3] = list[(ix + LX + skew) % LX][LY - 1];
        nn[N + ix - LX][1] = list[(ix + LX - skew) % LX][0];
      }
    }
  }

  int index(int x, int y) const {
    int y_offset = 0;
    if (y >= LY) {
      y_offset = y / LY;
    } else if (y < 0) {
      y_offset = (y + 1) / LY - 1;
    }
    y -= LY * y_offset;
    x -= skew * y_offset;
    x %= LX;
    if (x < 0) x += LX;
    return list[x][y];
  }
  int left(int i) const { return nn[i][0]; }
  int top(int i) const { return nn[i][1]; }
  int right(int i) const { return nn[i][2]; }
  int bottom(int i) const { return nn[i][3]; }
  int neighbor(int i, int d) const { return nn[i][d]; }
  int other(int i, int dx, int dy) const {
    while (dx != 0) {
      if (dx > 0) {
        i = right(i);
        --dx;
      } else {
        i = left(i);
        ++dx;
      }
    }
    while (dy != 0) {
      if (dy > 0) {
        i = top(i);
        --dy;
      } else {
        i = bottom(i);
        ++dy;
      }
    }
    return i;
  }

  // SquareLattice::check_dims (SquareLattice.cpp:216-238): bond dims match.
  void check_dims() const {
    for (int i = 0; i < N; ++i) {
      if (pdim[i] <= 0) fail(TG_E_INPUT, "physical_dim of site " + std::to_string(i) + " not set");
      for (int l = 0; l < 4; ++l)
        if (vdim[i][l] <= 0)
          fail(TG_E_INPUT, "virtual_dim of site " + std::to_string(i) + " not set");
      const int r = right(i), t = top(i);
      if (vdim[i][2] != vdim[r][0])
        fail(TG_E_INPUT, "virtual_dim mismatch between site " + std::to_string(i) + " and its right neighbour");
      if (vdim[i][1] != vdim[t][3])
        fail(TG_E_INPUT, "virtual_dim mismatch between site " + std::to_string(i) + " and its top neighbour");
    }
  }
};

}  // namespace tg
