// Stand-ins for the Cubism types that the reference's hot-path sources name
// (grid, block info, block lab with periodic ghosts, synchronizer), written
// for compiling those sources unmodified on one process. Test infrastructure
// of the oracle only: the Cubism submodule itself is absent from the
// reference snapshot, and nothing here is its code. Only what the reference's
// uniform periodic path calls is functional; the rest exists to compile.
#pragma once
#include <mpi.h>
#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <cassert>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace cubism {

struct BlockInfo {
  long long blockID = 0;
  int index[3] = {0, 0, 0};
  double origin[3] = {0, 0, 0};
  double h = 0, h_gridpoint = 0;
  double uniform_grid_spacing[3] = {0, 0, 0};
  void* ptrBlock = nullptr;
  void* auxiliary = nullptr;
  bool special = false;
  template <typename T>
  void pos(T p[3], int ix, int iy, int iz) const {
    p[0] = origin[0] + h_gridpoint * (ix + 0.5);
    p[1] = origin[1] + h_gridpoint * (iy + 0.5);
    p[2] = origin[2] + h_gridpoint * (iz + 0.5);
  }
  template <typename T>
  std::array<T, 3> pos(int ix, int iy, int iz) const {
    std::array<T, 3> p;
    pos(p.data(), ix, iy, iz);
    return p;
  }
  template <typename T>
  void spacing(T s[3], int, int, int) const {
    s[0] = s[1] = s[2] = h_gridpoint;
  }
};

struct StencilInfo {
  int sx = 0, sy = 0, sz = 0, ex = 1, ey = 1, ez = 1;
  bool tensorial = false;
  std::vector<int> selcomponents;
  StencilInfo() = default;
  StencilInfo(int _sx, int _sy, int _sz, int _ex, int _ey, int _ez, bool t, const std::vector<int>& c)
      : sx(_sx), sy(_sy), sz(_sz), ex(_ex), ey(_ey), ez(_ez), tensorial(t), selcomponents(c) {}
};

class Profiler;
class ArgumentParser;
namespace SliceTypesMPI {
template <typename grid_t>
class Slice {};
}  // namespace SliceTypesMPI

// The set of blocks a compute() pass visits (one process: all of them).
template <typename TReal>
class SynchronizerMPI {
 public:
  std::vector<BlockInfo> inner;
  std::vector<BlockInfo> avail_inner() { return inner; }
  std::vector<BlockInfo> avail_halo() { return {}; }
};

// Uniform grid of bpd[0] x bpd[1] x bpd[2] blocks, x fastest, periodic.
template <typename TBlock, template <typename> class allocator = std::allocator>
class Grid {
 public:
  typedef TBlock BlockType;
  typedef typename TBlock::ElementType ElementType;
  static constexpr size_t kAlign = 64;  // CUBISM_ALIGNMENT: blocks hold 32-byte aligned members
  std::vector<TBlock*> blocks;
  std::vector<BlockInfo> infos;
  int bpd[3] = {1, 1, 1};
  double h = 1;
  Grid() = default;
  Grid(int bx, int by, int bz, double hh) { setup(bx, by, bz, hh); }
  ~Grid() {
    for (TBlock* b : blocks) ::operator delete(static_cast<void*>(b), std::align_val_t(kAlign));
  }
  void setup(int bx, int by, int bz, double hh) {
    bpd[0] = bx, bpd[1] = by, bpd[2] = bz, h = hh;
    const int nb = bx * by * bz;
    blocks.resize(nb);
    infos.resize(nb);
    for (int i = 0; i < nb; ++i) {
      void* mem = ::operator new(sizeof(TBlock), std::align_val_t(kAlign));
      std::memset(mem, 0, sizeof(TBlock));
      blocks[i] = static_cast<TBlock*>(mem);
      BlockInfo& I = infos[i];
      I.blockID = i;
      I.index[0] = i % bx;
      I.index[1] = (i / bx) % by;
      I.index[2] = i / (bx * by);
      for (int d = 0; d < 3; ++d) {
        I.origin[d] = I.index[d] * TBlock::sizeX * hh;
        I.uniform_grid_spacing[d] = hh;
      }
      I.h = I.h_gridpoint = hh;
      I.ptrBlock = blocks[i];
    }
  }
  std::vector<BlockInfo>& getBlocksInfo() { return infos; }
  const std::vector<BlockInfo>& getBlocksInfo() const { return infos; }
  std::vector<BlockInfo>& getResidentBlocksInfo() { return infos; }
  const std::vector<BlockInfo>& getResidentBlocksInfo() const { return infos; }
  int getBlocksPerDimension(int d) const { return bpd[d]; }
  int getResidentBlocksPerDimension(int d) const { return bpd[d]; }
  TBlock& operator()(int ix, int iy, int iz) const {
    auto w = [](int i, int n) { return ((i % n) + n) % n; };
    return *blocks[(w(iz, bpd[2]) * bpd[1] + w(iy, bpd[1])) * bpd[0] + w(ix, bpd[0])];
  }
  double getH() const { return h; }
};

template <typename TGrid>
class GridMPI : public TGrid {
 public:
  typedef typename TGrid::BlockType BlockType;
  using TGrid::TGrid;
  GridMPI() = default;
  // (processes per dimension, blocks per process and dimension, the longest
  // side): one process, so the grid is the processes' blocks, with
  // h = maxextent / (cells along the longest dimension)
  GridMPI(int npx, int npy, int npz, int bx, int by, int bz, double maxextent, MPI_Comm) {
    const int mx = std::max({bx * npx, by * npy, bz * npz});
    this->setup(bx * npx, by * npy, bz * npz, maxextent / (mx * TGrid::BlockType::sizeX));
  }
  SynchronizerMPI<double> synch;
  MPI_Comm getCartComm() const { return MPI_COMM_WORLD; }
  MPI_Comm getWorldComm() const { return MPI_COMM_WORLD; }
  template <typename Processing>
  SynchronizerMPI<double>& sync(const Processing&) {
    synch.inner = this->infos;
    return synch;
  }
};

// Cached block with ghosts [start, size + end - 1) per direction.
// (Elements are plain aggregates of Reals without a default constructor; as
// in Cubism, block and lab storage is raw memory used in place.)
template <typename E>
struct LabCache {
  std::vector<double> raw;
  int W[3] = {0, 0, 0};
  void resize(int wx, int wy, int wz) {
    W[0] = wx, W[1] = wy, W[2] = wz;
    raw.assign(((size_t)wx * wy * wz * sizeof(E) + sizeof(double) - 1) / sizeof(double), 0.0);
  }
  E* d() { return reinterpret_cast<E*>(raw.data()); }
  const E* d() const { return reinterpret_cast<const E*>(raw.data()); }
  E& Access(int ix, int iy, int iz) { return d()[((size_t)iz * W[1] + iy) * W[0] + ix]; }
  const E& Access(int ix, int iy, int iz) const { return d()[((size_t)iz * W[1] + iy) * W[0] + ix]; }
};

// Block lab with periodic ghosts taken from the neighbouring blocks (edges and
// corners included), stencil width from the kernel's StencilInfo.
template <typename TBlock, template <typename> class allocator = std::allocator>
class BlockLab {
 public:
  typedef typename TBlock::ElementType ElementType;

 protected:
  LabCache<ElementType>* m_cacheBlock = nullptr;
  int m_stencilStart[3] = {-1, -1, -1};
  int m_stencilEnd[3] = {2, 2, 2};
  int NX = 1, NY = 1, NZ = 1;
  const void* m_grid = nullptr;
  TBlock& (*m_fetch)(const void*, int, int, int) = nullptr;
  LabCache<ElementType> m_cache;

 public:
  BlockLab() { m_cacheBlock = &m_cache; }
  virtual ~BlockLab() = default;
  template <typename TGrid, typename TSynch>
  void prepare(TGrid& grid, TSynch&) {
    prepare_grid(grid, StencilInfo(-1, -1, -1, 2, 2, 2, true, {}));
  }
  template <typename TGrid>
  void prepare_grid(TGrid& grid, const StencilInfo& st) {
    m_stencilStart[0] = st.sx, m_stencilStart[1] = st.sy, m_stencilStart[2] = st.sz;
    m_stencilEnd[0] = st.ex, m_stencilEnd[1] = st.ey, m_stencilEnd[2] = st.ez;
    NX = grid.getBlocksPerDimension(0), NY = grid.getBlocksPerDimension(1), NZ = grid.getBlocksPerDimension(2);
    m_grid = &grid;
    m_fetch = [](const void* g, int x, int y, int z) -> TBlock& { return (*static_cast<const TGrid*>(g))(x, y, z); };
    m_cache.resize(TBlock::sizeX + st.ex - st.sx - 1, TBlock::sizeY + st.ey - st.sy - 1,
                   TBlock::sizeZ + st.ez - st.sz - 1);
  }
  void load(const BlockInfo& info, const double = 0, const bool = false) {
    const int S[3] = {TBlock::sizeX, TBlock::sizeY, TBlock::sizeZ};
    for (int iz = m_stencilStart[2]; iz < S[2] + m_stencilEnd[2] - 1; ++iz)
      for (int iy = m_stencilStart[1]; iy < S[1] + m_stencilEnd[1] - 1; ++iy)
        for (int ix = m_stencilStart[0]; ix < S[0] + m_stencilEnd[0] - 1; ++ix) {
          const int g[3] = {info.index[0] * S[0] + ix, info.index[1] * S[1] + iy, info.index[2] * S[2] + iz};
          int b[3], c[3];
          for (int d = 0; d < 3; ++d) {
            b[d] = g[d] >= 0 ? g[d] / S[d] : -((-g[d] + S[d] - 1) / S[d]);
            c[d] = g[d] - b[d] * S[d];
          }
          const TBlock& blk = m_fetch(m_grid, b[0], b[1], b[2]);
          m_cache.Access(ix - m_stencilStart[0], iy - m_stencilStart[1], iz - m_stencilStart[2]) = blk(c[0], c[1], c[2]);
        }
    static_cast<void>(info);
  }
  ElementType& operator()(int ix, int iy = 0, int iz = 0) {
    return m_cache.Access(ix - m_stencilStart[0], iy - m_stencilStart[1], iz - m_stencilStart[2]);
  }
  const ElementType& operator()(int ix, int iy = 0, int iz = 0) const {
    return m_cache.Access(ix - m_stencilStart[0], iy - m_stencilStart[1], iz - m_stencilStart[2]);
  }
  ElementType& read(int ix, int iy = 0, int iz = 0) { return (*this)(ix, iy, iz); }
};

template <typename TLab>
class BlockLabMPI : public TLab {};

}  // namespace cubism
