// Host-side unstructured mesh: connectivity, geometry and least-squares
// gradient weights, computed once per mesh in FP64 with the same operation
// order as the reference so that every derived integer array is identical
// and every derived floating-point value rounds identically.
#pragma once

#include <string>
#include <vector>

#include "common.hpp"

namespace fvm {

struct FaceGroup {
  int id = 0;
  int offset = 0;  // first face of the group
  int size = 0;
  std::string type;  // "interior", "wall", "symmetry", "velocity-inlet", ...
};

struct HostMesh {
  // ---- inputs (Mesh 7-argument constructor, reference Mesh.cpp:132-247)
  int dim = 0;
  int nCells = 0;   // self cells
  int nGhost = 0;   // one ghost cell per boundary face
  int nNodes = 0;
  int nFaces = 0;
  std::vector<double> xyz;       // 3 * nNodes
  std::vector<int> faceCells;    // 2 * nFaces: (c0, c1); c1 of a boundary face is a ghost
  CSR faceNodes;                 // nFaces rows
  std::vector<FaceGroup> groups; // groups[0] is the interior group

  // ---- connectivity (reference CRConnectivity.cpp:73-94,167-270,730-790)
  CSR cellFaces;                 // (nCells + nGhost) rows, faces ascending
  CSR cellCells;                 // (nCells + nGhost) rows, reference column order
  std::vector<int> pairToCol;    // 2 * nFaces: position of c1 in row c0, of c0 in row c1

  // ---- geometry (reference MeshMetricsCalculator_impl.h)
  std::vector<double> faceArea;      // 3 * nFaces
  std::vector<double> faceAreaMag;   // nFaces
  std::vector<double> faceCentroid;  // 3 * nFaces
  std::vector<double> cellCentroid;  // 3 * (nCells + nGhost)
  std::vector<double> cellVolume;    // nCells + nGhost

  // ---- least-squares gradient weights, 3 per cellCells entry
  // (reference GradientModel.h:126-436)
  std::vector<double> gradCoeff;

  int nTotalCells() const { return nCells + nGhost; }
  int nInteriorFaces() const { return groups.empty() ? 0 : groups[0].size; }
  bool isBoundaryGroupType(const std::string& t) const {
    return t != "interior" && t != "interface" && t != "dielectric interface";
  }

  // Validates the inputs and computes everything above.
  void build();

 private:
  void buildConnectivity();
  void buildGeometry();
  void buildGradientWeights();
};

// Builds the mesh from the reference constructor's arrays. faceNodes holds
// the nodes of every face back to back; faceNodeCount their counts;
// groupSize the face count of the interior group followed by each boundary
// group. Boundary groups get ids 1..k and type "wall", as the reference's
// constructor assigns them.
HostMesh* make_mesh(int dim, int nCells, int nNodes, const double* xyz, int nFaces,
                    const int* faceCells, const int* faceNodes, const int* faceNodeCount,
                    int nGroups, const int* groupSize);

}  // namespace fvm
