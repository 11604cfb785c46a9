// DOF classification and per-level index data of the HIF factorization.
//
// Closed-form restatement of the reference's partition code
// (arbenson/HIFDE3D src/Factor.cpp:313-755) over a frozen "remaining DOF"
// mask; produces the exact index lists the reference builds, in the same order.
#pragma once

#include <cstdint>
#include <vector>

namespace hif {

// include/data.hpp:6 (enum Face {TOP=0, BOTTOM, RIGHT, LEFT, FRONT, BACK}).
enum FaceId { TOP = 0, BOTTOM = 1, RIGHT = 2, LEFT = 3, FRONT = 4, BACK = 5 };

struct Partitioner {
  int N, P, NC;
  const uint8_t* rem;  // NC^3, DOF id i + NC j + NC^2 k

  int width(int level) const { return (1 << level) * P; }
  long long lin(int i, int j, int k) const {
    return i + (long long)NC * j + (long long)NC * NC * k;
  }
  // IsInterior, src/Factor.cpp:314-320.
  bool interior(int w, int a) const { return a > 0 && a <= N && (a % w) != 0; }
  bool remaining(int i, int j, int k) const { return rem[lin(i, j, k)] != 0; }

  // Cell box [lo, hi] per axis (src/Factor.cpp:366-367).
  void box(int w, const int c[3], int lo[3], int hi[3]) const {
    for (int a = 0; a < 3; ++a) {
      lo[a] = w * c[a] > 1 ? w * c[a] : 1;
      hi[a] = w * (c[a] + 1) < N ? w * (c[a] + 1) : N;
    }
  }

  // InteriorCellIndexData (src/Factor.cpp:359-392): global ids in i -> j -> k
  // scan order, positions of cell-interior (red) and face-interior (skel) DOFs.
  void cell_index(int level, const int c[3], std::vector<int>& global, std::vector<int>& red,
                  std::vector<int>& skel) const {
    const int w = width(level);
    int lo[3], hi[3];
    box(w, c, lo, hi);
    global.clear();
    red.clear();
    skel.clear();
    for (int i = lo[0]; i <= hi[0]; ++i) {
      const bool ai = interior(w, i);
      for (int j = lo[1]; j <= hi[1]; ++j) {
        const bool aj = interior(w, j);
        for (int k = lo[2]; k <= hi[2]; ++k) {
          if (!remaining(i, j, k)) continue;
          const bool ak = interior(w, k);
          const int cnt = (int)ai + (int)aj + (int)ak;
          if (cnt == 3) {
            red.push_back((int)global.size());
            global.push_back((int)lin(i, j, k));
          } else if (cnt == 2) {
            skel.push_back((int)global.size());
            global.push_back((int)lin(i, j, k));
          }
        }
      }
    }
  }

  // Scan plane of InteriorFaceDOFs / InteriorEdgeDOFs (src/Factor.cpp:402-643).
  // Returns false when the reference returns early ("no face"). The FRONT
  // test of the reference compares with 0 (src/Factor.cpp:486), which never
  // holds, so a cell on the k = 1 plane scans that plane; reproduced.
  bool face_plane(int level, const int c[3], int face, int lo_out[3], int hi_out[3]) const {
    const int w = width(level);
    int lo[3], hi[3];
    box(w, c, lo, hi);
    for (int a = 0; a < 3; ++a) {
      lo_out[a] = lo[a];
      hi_out[a] = hi[a];
    }
    switch (face) {
      case TOP:
        if (lo[0] == 1) return false;
        hi_out[0] = lo[0];
        return true;
      case BOTTOM:
        if (hi[0] == N) return false;
        lo_out[0] = hi[0];
        return true;
      case LEFT:
        if (lo[1] == 1) return false;
        hi_out[1] = lo[1];
        return true;
      case RIGHT:
        if (hi[1] == N) return false;
        lo_out[1] = hi[1];
        return true;
      case FRONT:
        if (lo[2] == 0) return false;
        hi_out[2] = lo[2];
        return true;
      case BACK:
        if (hi[2] == N) return false;
        lo_out[2] = hi[2];
        return true;
    }
    return false;
  }

  // Appends the remaining face-interior (edge == false) or edge-interior
  // (edge == true) DOFs of a face plane, in the reference's scan order.
  void plane_dofs(int level, const int c[3], int face, bool edge, std::vector<int>& out) const {
    int lo[3], hi[3];
    if (!face_plane(level, c, face, lo, hi)) return;
    const int w = width(level);
    for (int i = lo[0]; i <= hi[0]; ++i) {
      const bool ai = interior(w, i);
      for (int j = lo[1]; j <= hi[1]; ++j) {
        const bool aj = interior(w, j);
        for (int k = lo[2]; k <= hi[2]; ++k) {
          const bool ak = interior(w, k);
          const int cnt = (int)ai + (int)aj + (int)ak;
          if ((edge ? cnt == 1 : cnt == 2) && remaining(i, j, k))
            out.push_back((int)lin(i, j, k));
        }
      }
    }
  }

  // SkelInteractionIndexData (src/Factor.cpp:645-755) for TOP, LEFT, FRONT.
  // Returns false if the face does not exist. nbr receives the neighbour cell.
  bool skel_interaction(int level, const int c[3], int face, std::vector<int>& rows,
                        std::vector<int>& cols, int nbr[3]) const {
    const int w = width(level);
    int lo[3], hi[3];
    box(w, c, lo, hi);
    rows.clear();
    cols.clear();
    int own[5], nbf[5], axis;
    if (face == TOP) {
      if (lo[0] == 1) return false;
      const int o[5] = {BOTTOM, LEFT, RIGHT, FRONT, BACK}, q[5] = {TOP, LEFT, RIGHT, FRONT, BACK};
      for (int t = 0; t < 5; ++t) { own[t] = o[t]; nbf[t] = q[t]; }
      axis = 0;
    } else if (face == LEFT) {
      if (lo[1] == 1) return false;
      const int o[5] = {TOP, BOTTOM, RIGHT, FRONT, BACK}, q[5] = {TOP, BOTTOM, LEFT, FRONT, BACK};
      for (int t = 0; t < 5; ++t) { own[t] = o[t]; nbf[t] = q[t]; }
      axis = 1;
    } else if (face == FRONT) {
      if (lo[2] == 1) return false;
      const int o[5] = {TOP, BOTTOM, LEFT, RIGHT, BACK}, q[5] = {TOP, BOTTOM, LEFT, RIGHT, FRONT};
      for (int t = 0; t < 5; ++t) { own[t] = o[t]; nbf[t] = q[t]; }
      axis = 2;
    } else {
      return false;
    }
    plane_dofs(level, c, face, false, cols);
    plane_dofs(level, c, face, true, rows);
    for (int t = 0; t < 5; ++t) plane_dofs(level, c, own[t], false, rows);
    for (int a = 0; a < 3; ++a) nbr[a] = c[a];
    nbr[axis] -= 1;
    for (int t = 0; t < 5; ++t) plane_dofs(level, nbr, nbf[t], false, rows);
    return true;
  }
};

}  // namespace hif
