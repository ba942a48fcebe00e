// Fluent case-file (.cas) import into the arrays of the 7-argument Mesh
// constructor: the reference's FluentReader::readMesh + getMeshList
// (src/modules/importers/FluentReader.cpp:572-611, 696-952, 954-1040),
// written from the file format.
//
// A case file is a sequence of parenthesised sections "(id ...)": 2 the
// dimension, 10 nodes, 12 cells, 13 faces, 18 periodic face pairs, 39/45
// zone names and types; ids 20xx / 30xx hold the same data in binary
// (single / double precision), ending with "End of Binary Section id)".
// Headers are hexadecimal; ASCII bodies too, except node coordinates.
#pragma once

#include <map>
#include <string>
#include <vector>

namespace fvm {

struct FluentMeshArrays {
  int dim = 0;
  int nCells = 0;                  // cells of the zone (self cells)
  std::vector<double> xyz;         // 3 per node (z = 0 in 2D)
  std::vector<int> faceCells;      // 2 per face; boundary faces: (cell, nCells + k)
  std::vector<int> faceNodes;      // per face, in the face's node order
  std::vector<int> faceNodeCount;
  std::vector<int> groupSize;      // interior faces, then one entry per boundary zone
  std::vector<int> groupId;        // Fluent zone id of each group (0 for the interior)
  std::vector<std::string> groupType;  // "interior", then the zones' type names
};

class FluentCase {
 public:
  // Reads and parses the whole file; throws fvm::Error on malformed input
  // or on what this import does not cover (periodic face pairs, faces
  // between two cell zones).
  explicit FluentCase(const std::string& path);
  int dimension() const { return dim_; }
  int numCellZones() const { return (int)cellZones_.size(); }
  // Mesh of the k-th cell zone (ascending zone id), as getMeshList()[k].
  FluentMeshArrays mesh(int k) const;

 private:
  struct CellZone {
    int id, first, last, type;  // 0-based cells first..last
  };
  struct FaceZone {
    int id, first, last, bcType;  // 0-based faces first..last
    std::string name, kind;
  };
  int dim_ = 0;
  int numNodes_ = 0, numCells_ = 0, numFaces_ = 0;
  std::vector<double> xyz_;
  std::map<int, CellZone> cellZones_;
  std::map<int, FaceZone> faceZones_;
  std::map<int, std::pair<std::string, std::string>> zoneNames_;  // id -> (type, name)
  std::vector<int> fnPtr_, fnIdx_;  // global face -> global nodes, file order, 0-based
  std::vector<int> fnOrder_;        // faces in the order their nodes were read
  std::vector<int> c0_, c1_;        // Fluent cell numbers (1-based; 0: none)
  std::vector<char> faceSeen_;
  bool periodic_ = false;
  int zoneOfCell(int c) const;      // cell zone id of a 0-based cell, or 0
};

}  // namespace fvm
