// Force-included when compiling the reference Mesh.cpp for the CPU oracle.
// The reference's KSearchTree wraps CGAL (absent here) and is used only by
// mesh-assembly helpers that the thermal path never calls; this stub takes
// its include guard and provides the same member names, each of which
// throws if reached.
#ifndef _KSEARCHTREE_H_
#define _KSEARCHTREE_H_
#include <stdexcept>
#include <vector>
#include "Vector.h"
#include "Array.h"
class KSearchTree {
 public:
  typedef Vector<double, 3> Vec3D;
  KSearchTree() {}
  explicit KSearchTree(const Array<Vec3D>&) {}
  void insert(const Vec3D&, int) { fail(); }
  void findNeighbors(const Vec3D&, int, Array<int>&) { fail(); }
 private:
  static void fail() { throw std::runtime_error("KSearchTree is not available in the oracle build"); }
};
#endif
