// Fluent case-file import (see fluent.hpp).
#include "fluent.hpp"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>

#include "common.hpp"

namespace fvm {

namespace {

constexpr int kPeriodicShadow = 8;  // face thread type of a periodic shadow zone

// Position in the file's bytes with the few moves the format needs.
struct Cursor {
  const std::string& s;
  size_t p = 0;
  explicit Cursor(const std::string& buf) : s(buf) {}

  bool eof() const { return p >= s.size(); }
  // just past the next '(' (whatever the nesting); false at the end
  bool open() {
    while (p < s.size())
      if (s[p++] == '(') return true;
    return false;
  }
  // just past the ')' that closes the current list; nested lists skipped
  void close() {
    int depth = 0;
    while (p < s.size()) {
      const char c = s[p++];
      if (c == '(') {
        depth++;
      } else if (c == ')') {
        if (depth == 0) return;
        depth--;
      }
    }
  }
  void space() {
    while (p < s.size() && std::isspace((unsigned char)s[p])) p++;
  }
  bool number(int& v, int base) {
    space();
    if (eof()) return false;
    const char* b = s.c_str() + p;
    char* e = nullptr;
    const long x = std::strtol(b, &e, base);
    if (e == b) return false;
    p += (size_t)(e - b);
    v = (int)x;
    return true;
  }
  bool dec(int& v) { return number(v, 10); }
  bool hex(int& v) { return number(v, 16); }
  double real() {
    space();
    const char* b = s.c_str() + p;
    char* e = nullptr;
    const double x = std::strtod(b, &e);
    FVM_REQUIRE(e != b, kBadMesh, "Fluent file: expected a number at byte " + std::to_string(p));
    p += (size_t)(e - b);
    return x;
  }
  std::string token() {
    space();
    const size_t b = p;
    while (p < s.size() && !std::isspace((unsigned char)s[p]) && s[p] != '(' && s[p] != ')') p++;
    return s.substr(b, p - b);
  }
  template <class T>
  T binary() {
    FVM_REQUIRE(p + sizeof(T) <= s.size(), kBadMesh, "Fluent file: binary section ends early");
    T v;
    std::memcpy(&v, s.data() + p, sizeof(T));
    p += sizeof(T);
    return v;
  }
  int integer(bool bin) {
    if (bin) return binary<int>();
    int v = 0;
    FVM_REQUIRE(hex(v), kBadMesh, "Fluent file: expected a hexadecimal integer at byte " + std::to_string(p));
    return v;
  }
  // past the "End of Binary Section <id>)" that ends a binary section
  void closeBinary(int id) {
    static const char kMark[] = "End of Binary Section";
    const size_t q = s.find(kMark, p);
    FVM_REQUIRE(q != std::string::npos, kBadMesh,
                "Fluent file: binary section " + std::to_string(id) + " is not terminated");
    p = q + sizeof(kMark) - 1;
    int got = 0;
    dec(got);
    FVM_REQUIRE(got == id, kBadMesh,
                "Fluent file: binary section " + std::to_string(id) + " closed as " + std::to_string(got));
    close();
  }
  // a section header "(a b c d [e])" in hexadecimal; e = -1 when absent
  void header(int v[5]) {
    FVM_REQUIRE(open(), kBadMesh, "Fluent file: missing section header");
    for (int k = 0; k < 4; k++)
      FVM_REQUIRE(hex(v[k]), kBadMesh, "Fluent file: malformed section header at byte " + std::to_string(p));
    if (!hex(v[4])) v[4] = -1;
    close();
  }
};

}  // namespace

FluentCase::FluentCase(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  FVM_REQUIRE(in.good(), kBadArgument, "cannot open Fluent case file " + path);
  const std::string buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  Cursor c(buf);
  while (c.open()) {
    int id = 0;
    if (!c.dec(id)) {
      c.close();
      continue;
    }
    const bool bin = id > 1000;
    const bool dp = id > 3000;
    const int kind = id % 1000;
    int h[5];
    switch (kind) {
      case 2:
        FVM_REQUIRE(c.dec(dim_) && (dim_ == 2 || dim_ == 3), kBadMesh, "Fluent file: bad dimension");
        c.close();
        break;
      case 10: {  // nodes
        c.header(h);
        const int zone = h[0], first = h[1], last = h[2];
        if (zone == 0) {
          numNodes_ = last;
          xyz_.assign(3 * (size_t)std::max(numNodes_, 0), 0.0);
          c.close();
          break;
        }
        FVM_REQUIRE(dim_ > 0, kBadMesh, "Fluent file: nodes before the dimension");
        FVM_REQUIRE(first >= 1 && last <= numNodes_ && first <= last + 1, kBadMesh,
                    "Fluent file: node range outside the declared nodes");
        FVM_REQUIRE(c.open(), kBadMesh, "Fluent file: node section without data");
        for (int i = first; i <= last; i++)
          for (int d = 0; d < dim_; d++)
            xyz_[3 * (size_t)(i - 1) + d] = bin ? (dp ? c.binary<double>() : (double)c.binary<float>()) : c.real();
        if (bin) {
          c.closeBinary(id);
        } else {
          c.close();
          c.close();
        }
        break;
      }
      case 12: {  // cells
        c.header(h);
        const int zone = h[0], first = h[1], last = h[2], type = h[3];
        if (zone == 0) {
          numCells_ = last;
        } else if (type == 1 || type == 17) {
          cellZones_[zone] = CellZone{zone, first - 1, last - 1, type};
        } else if (type == 32) {
          numCells_ -= last - first + 1;  // dead cells
        } else {
          throw Error(kUnsupported, "Fluent file: cell thread type " + std::to_string(type) + " not handled");
        }
        if (zone != 0 && bin)
          c.closeBinary(id);
        else
          c.close();
        break;
      }
      case 13: {  // faces
        c.header(h);
        const int zone = h[0], first = h[1], last = h[2], type = h[3];
        int shape = h[4];
        if (zone == 0) {
          numFaces_ = last;
          c0_.assign(std::max(numFaces_, 0), 0);
          c1_.assign(std::max(numFaces_, 0), 0);
          faceSeen_.assign(std::max(numFaces_, 0), 0);
          fnPtr_.assign((size_t)std::max(numFaces_, 0) + 1, 0);
          c.close();
          break;
        }
        if (type == 0 || type == 31) {  // hanging / parent faces: not part of the mesh
          if (bin)
            c.closeBinary(id);
          else
            c.close();
          break;
        }
        FVM_REQUIRE(first >= 1 && last <= numFaces_ && first <= last + 1, kBadMesh,
                    "Fluent file: face range outside the declared faces");
        if (shape < 0) shape = dim_;
        faceZones_[zone] = FaceZone{zone, first - 1, last - 1, type, "", ""};
        FVM_REQUIRE(c.open(), kBadMesh, "Fluent file: face section without data");
        std::vector<int> nodes;
        for (int f = first - 1; f < last; f++) {
          int nn = shape;
          if (shape == 0 || shape == 5) nn = c.integer(bin);
          FVM_REQUIRE(nn >= 2 && nn <= 64, kBadMesh, "Fluent file: face with " + std::to_string(nn) + " nodes");
          nodes.resize(nn);
          for (int k = 0; k < nn; k++) {
            nodes[k] = c.integer(bin) - 1;
            FVM_REQUIRE(nodes[k] >= 0 && nodes[k] < numNodes_, kBadMesh, "Fluent file: face node out of range");
          }
          c0_[f] = c.integer(bin);
          c1_[f] = c.integer(bin);
          FVM_REQUIRE(c0_[f] >= 0 && c0_[f] <= numCells_ && c1_[f] >= 0 && c1_[f] <= numCells_, kBadMesh,
                      "Fluent file: face cell out of range");
          FVM_REQUIRE(!faceSeen_[f], kBadMesh, "Fluent file: face defined twice");
          faceSeen_[f] = 1;
          fnPtr_[f + 1] = nn;
          // nodes kept by face; the CSR is assembled once all zones are read
          fnIdx_.insert(fnIdx_.end(), nodes.begin(), nodes.end());
          fnOrder_.push_back(f);
        }
        if (bin) {
          c.closeBinary(id);
        } else {
          c.close();
          c.close();
        }
        break;
      }
      case 18:  // periodic face pairs
        periodic_ = true;
        if (bin)
          c.closeBinary(id);
        else
          c.close();
        break;
      case 39:
      case 45: {  // zone type and name
        FVM_REQUIRE(c.open(), kBadMesh, "Fluent file: malformed zone section");
        int zid = 0;
        FVM_REQUIRE(c.dec(zid), kBadMesh, "Fluent file: malformed zone id");
        std::string type = c.token();
        std::string name = c.token();
        std::replace(name.begin(), name.end(), '-', '_');
        zoneNames_[zid] = {type, name};
        c.close();  // the zone's header list
        c.close();  // the section
        break;
      }
      default:
        if (bin)
          c.closeBinary(id);
        else
          c.close();
    }
  }
  FVM_REQUIRE(dim_ == 2 || dim_ == 3, kBadMesh, "Fluent file: no dimension section");
  FVM_REQUIRE(!cellZones_.empty(), kBadMesh, "Fluent file: no cell zone");
  // face -> nodes CSR in face order (sections may come in any order)
  std::vector<int> start((size_t)numFaces_, -1);
  {
    size_t o = 0;
    for (int f : fnOrder_) {
      start[f] = (int)o;
      o += fnPtr_[f + 1];
    }
  }
  std::vector<int> ptr((size_t)numFaces_ + 1, 0), idx;
  for (int f = 0; f < numFaces_; f++) ptr[f + 1] = ptr[f] + fnPtr_[f + 1];
  idx.resize(ptr[numFaces_]);
  for (int f = 0; f < numFaces_; f++)
    if (start[f] >= 0) std::copy(fnIdx_.begin() + start[f], fnIdx_.begin() + start[f] + fnPtr_[f + 1], idx.begin() + ptr[f]);
  fnPtr_ = std::move(ptr);
  fnIdx_ = std::move(idx);
  for (auto& kv : faceZones_) {
    auto it = zoneNames_.find(kv.first);
    if (it != zoneNames_.end()) {
      kv.second.kind = it->second.first;
      kv.second.name = it->second.second;
    }
  }
}

int FluentCase::zoneOfCell(int c) const {
  for (const auto& kv : cellZones_)
    if (c >= kv.second.first && c <= kv.second.last) return kv.first;
  return 0;
}

FluentMeshArrays FluentCase::mesh(int k) const {
  FVM_REQUIRE(k >= 0 && k < (int)cellZones_.size(), kBadArgument, "no such cell zone");
  FVM_REQUIRE(!periodic_, kUnsupported, "Fluent import: periodic face pairs are not supported");
  auto zit = cellZones_.begin();
  std::advance(zit, k);
  const CellZone& cz = zit->second;
  const int nCells = cz.last - cz.first + 1;
  // the interior-side cell of a face (0-based) and whether it has a ghost
  auto inner = [&](int f) { return c0_[f] != 0 ? c0_[f] - 1 : c1_[f] - 1; };
  auto outer = [&](int f) { return (c0_[f] != 0 && c1_[f] != 0) ? c1_[f] - 1 : -1; };
  std::vector<int> interiorZones, boundaryZones;
  for (const auto& kv : faceZones_) {
    const FaceZone& fz = kv.second;
    if (fz.last < fz.first) continue;
    const int f = fz.first;
    if (c0_[f] == 0 && c1_[f] == 0) continue;  // a boundary mesh without cells
    const int left = zoneOfCell(inner(f));
    if (left != cz.id) continue;
    const int o = outer(f);
    const int right = o >= 0 ? zoneOfCell(o) : 0;
    if (right == left) {
      interiorZones.push_back(fz.id);
    } else if (right > 0) {
      throw Error(kUnsupported, "Fluent import: faces between two cell zones (interfaces) are not supported");
    } else {
      FVM_REQUIRE(fz.kind != "interface", kUnsupported, "Fluent import: interface zones are not supported");
      boundaryZones.push_back(fz.id);
    }
  }
  FluentMeshArrays m;
  m.dim = dim_;
  m.nCells = nCells;
  std::vector<int> faces;
  for (int z : interiorZones) {
    const FaceZone& fz = faceZones_.at(z);
    for (int f = fz.first; f <= fz.last; f++) faces.push_back(f);
  }
  m.groupSize.push_back((int)faces.size());
  m.groupId.push_back(0);
  m.groupType.push_back("interior");
  for (int z : boundaryZones) {
    const FaceZone& fz = faceZones_.at(z);
    for (int f = fz.first; f <= fz.last; f++) faces.push_back(f);
    m.groupSize.push_back(fz.last - fz.first + 1);
    m.groupId.push_back(fz.id);
    m.groupType.push_back(fz.bcType == kPeriodicShadow ? std::string("shadow") : fz.kind);
  }
  const int F = (int)faces.size();
  // each face's nodes as the mesh stores them: Fluent orders them the other
  // way round in 3D, and a face whose first cell is missing turns over
  auto faceNodes = [&](int f, std::vector<int>& out) {
    bool reverse = dim_ == 3;
    if (c0_[f] == 0) reverse = !reverse;
    out.assign(fnIdx_.begin() + fnPtr_[f], fnIdx_.begin() + fnPtr_[f + 1]);
    if (reverse) std::reverse(out.begin(), out.end());
  };
  // cells of the zone -> their faces (ascending global face number)
  std::vector<int> cfPtr((size_t)nCells + 1, 0), cfIdx;
  for (int f = 0; f < numFaces_; f++) {
    if (!faceSeen_[f]) continue;
    for (int cc : {inner(f), outer(f)})
      if (cc >= cz.first && cc <= cz.last) cfPtr[cc - cz.first + 1]++;
  }
  for (int i = 0; i < nCells; i++) cfPtr[i + 1] += cfPtr[i];
  cfIdx.resize(cfPtr[nCells]);
  {
    std::vector<int> cur(cfPtr.begin(), cfPtr.end() - 1);
    for (int f = 0; f < numFaces_; f++) {
      if (!faceSeen_[f]) continue;
      const int a = inner(f), b = outer(f);
      if (a >= cz.first && a <= cz.last) cfIdx[cur[a - cz.first]++] = f;
      if (b != a && b >= cz.first && b <= cz.last) cfIdx[cur[b - cz.first]++] = f;
    }
  }
  // nodes numbered in first-visit order over the cells, their faces and
  // the faces' nodes
  std::vector<int> local((size_t)numNodes_, -1);
  std::vector<int> order;
  std::vector<int> tmp;
  for (int i = 0; i < nCells; i++)
    for (int q = cfPtr[i]; q < cfPtr[i + 1]; q++) {
      faceNodes(cfIdx[q], tmp);
      for (int v : tmp)
        if (local[v] < 0) {
          local[v] = (int)order.size();
          order.push_back(v);
        }
    }
  m.xyz.resize(3 * order.size());
  for (size_t v = 0; v < order.size(); v++)
    for (int d = 0; d < 3; d++) m.xyz[3 * v + d] = xyz_[3 * (size_t)order[v] + d];
  // faces: cells local, ghosts numbered after the cells in face order
  m.faceCells.resize(2 * (size_t)F);
  m.faceNodeCount.resize(F);
  int ghosts = 0;
  for (int q = 0; q < F; q++) {
    const int f = faces[q];
    const int a = inner(f), b = outer(f);
    m.faceCells[2 * q] = a - cz.first;
    m.faceCells[2 * q + 1] = b >= 0 ? b - cz.first : nCells + ghosts++;
    faceNodes(f, tmp);
    m.faceNodeCount[q] = (int)tmp.size();
    for (int v : tmp) {
      FVM_REQUIRE(local[v] >= 0, kBadMesh, "Fluent import: face node outside the zone's cells");
      m.faceNodes.push_back(local[v]);
    }
  }
  return m;
}

}  // namespace fvm
