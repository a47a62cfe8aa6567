// Crystal lattices (src/crystal.cpp:1-279, include/dft/types.hpp:51-86) and
// a device initialiser that places a Gaussian density peak on every site.
//
// The unit cells are the reference's (the same bases, cell dimensions in
// units of the nearest-neighbour distance, and the same x-fastest tiling
// order); the XYZ / CSV writers produce the reference's files.  The
// Gaussian-peak initialiser has no reference counterpart: it seeds a
// crystal density profile rho(r) = background + amplitude * sum_i
// exp(-alpha |r - R_i|^2) on the grid (z-fastest), with minimum-image
// periodic distances and the peaks cut where alpha r^2 > 40 (exp(-40) =
// 4e-18 of the peak height).
#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cdft_b200.h"
#include "cdft_common.cuh"

namespace cdft {
void set_last_error(const std::string& msg);
}  // namespace cdft

namespace {

using P3 = std::array<double, 3>;

constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kSqrt3 = 1.73205080756887729353;

// A unit cell: basis positions (fractions of the cell) and the cell edges.
struct Cell {
  std::vector<P3> basis;
  P3 dims;
};

const std::vector<P3>& bcc_basis() {
  static const std::vector<P3> b = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.5}};
  return b;
}

const std::vector<P3>& fcc_basis() {
  static const std::vector<P3> b = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};
  return b;
}

// Orientation indices 3..5 are the face diagonals 110, 101, 011: the two
// axes a diagonal lies in, and the axis normal to the face.
int face_normal(int orientation) { return orientation == CDFT_ORIENT_110 ? 2 : orientation == CDFT_ORIENT_101 ? 1 : 0; }

// crystal.cpp:80-200: the cell of a structure viewed along an orientation,
// with unit nearest-neighbour distance.
Cell unit_cell(int structure, int orientation) {
  if (orientation < CDFT_ORIENT_001 || orientation > CDFT_ORIENT_111) throw std::invalid_argument("unknown orientation");
  const bool axis = orientation <= CDFT_ORIENT_100;
  const bool face = orientation >= CDFT_ORIENT_110 && orientation <= CDFT_ORIENT_011;
  Cell c;
  switch (structure) {
    case CDFT_BCC: {
      const double a = 2.0 / kSqrt3;  // cube edge of unit nearest-neighbour distance
      if (axis) {
        c.basis = bcc_basis();
        c.dims = {a, a, a};
      } else if (face) {
        // the conventional cell seen along a face diagonal is a centred
        // cell sqrt(2) longer in the two in-face directions
        c.basis = fcc_basis();
        c.dims = {a, a, a};
        const int n = face_normal(orientation);
        for (int d = 0; d < 3; ++d)
          if (d != n) c.dims[d] *= kSqrt2;
      } else {
        c.basis = {{1.0 / 6, 0.5, 0.0},     {0.0, 0.0, 1.0 / 3},     {1.0 / 6, 0.5, 0.5},
                   {0.0, 0.0, 5.0 / 6},     {3.0 / 6, 0.5, 1.0 / 3}, {1.0 / 3, 0.0, 2.0 / 3},
                   {3.0 / 6, 0.5, 5.0 / 6}, {1.0 / 3, 0.0, 1.0 / 6}, {5.0 / 6, 0.5, 2.0 / 3},
                   {2.0 / 3, 0.0, 0.0},     {5.0 / 6, 0.5, 1.0 / 6}, {2.0 / 3, 0.0, 0.5}};
        c.dims = {2.0 * kSqrt2, 2.0 * std::sqrt(2.0 / 3.0), 2.0};
      }
      break;
    }
    case CDFT_FCC: {
      if (axis) {
        c.basis = fcc_basis();
        c.dims = {kSqrt2, kSqrt2, kSqrt2};
      } else if (face) {
        // along a face diagonal: a body-centred cell, sqrt(2) long on the
        // face normal
        c.basis = bcc_basis();
        c.dims = {1.0, 1.0, 1.0};
        c.dims[face_normal(orientation)] *= kSqrt2;
      } else {
        c.basis = {{0.0, 0.0, 0.0},         {0.5, 0.5, 0.0},         {0.5, 1.0 / 6, 1.0 / 3},
                   {0.0, 4.0 / 6, 1.0 / 3}, {0.0, 2.0 / 6, 2.0 / 3}, {0.5, 5.0 / 6, 2.0 / 3}};
        c.dims = {1.0, kSqrt3, std::sqrt(6.0)};
      }
      break;
    }
    case CDFT_HCP: {
      if (!axis) throw std::invalid_argument("HCP only supports orientations 001, 010, 100");
      c.basis = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.0, 2.0 / 6.0, 0.5}, {0.5, 5.0 / 6.0, 0.5}};
      c.dims = {1.0, kSqrt3, std::sqrt(8.0 / 3.0)};
      break;
    }
    default:
      throw std::invalid_argument("unknown crystal structure");
  }
  for (P3& b : c.basis)
    for (int d = 0; d < 3; ++d) b[d] *= c.dims[d];
  if (structure == CDFT_HCP && orientation != CDFT_ORIENT_001) {
    // crystal.cpp:47-73, 184-196: turn the c axis (z) onto y (010) or x
    // (100): the axis q in {y, x} takes z, z takes -q; positions wrap back
    // into the turned cell, whose edges q and z trade places
    const int q = orientation == CDFT_ORIENT_010 ? 1 : 0;
    P3 box = c.dims;
    std::swap(box[q], box[2]);
    for (P3& b : c.basis) {
      const double zq = b[2];
      b[2] = b[q];
      b[q] = -zq;
      for (int d = 0; d < 3; ++d) {
        b[d] = std::fmod(b[d], box[d]);
        if (b[d] < 0.0) b[d] += box[d];
      }
    }
    c.dims = box;
  }
  return c;
}

void check_shape(const long* shape) {
  if (!shape) throw std::invalid_argument("Shape must have exactly 3 elements");
  if (shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0)
    throw std::invalid_argument("Number of unit cells must be strictly positive in all directions");
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return CDFT_OK;
  } catch (const std::invalid_argument& e) {
    cdft::set_last_error(e.what());
    return CDFT_ERR_INVALID;
  } catch (const cdft::Error& e) {
    cdft::set_last_error(e.what());
    return e.code();
  } catch (const std::exception& e) {
    cdft::set_last_error(e.what());
    return CDFT_ERR_RUNTIME;
  }
}

constexpr double kPeakCut = 40.0;  // alpha r^2 beyond which a peak is dropped

struct PeakGrid {
  int nx, ny, nz;
  double dx;
  double L[3];
  int nb[3];       // bins per axis (edge >= the cut radius)
  double inv_bw[3];
  double alpha, amplitude, background;
};

// rho at each grid point: the sites in the point's bin and its neighbours
// (bins at least one cut radius wide hold every site within the cut), each
// at its minimum-image distance.  The bins are visited in a fixed order, so
// the sums are deterministic.
__global__ void k_gaussian_peaks(PeakGrid g, const double* __restrict__ sites, const int* __restrict__ bin_start,
                                 double* __restrict__ rho) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % g.nz);
    const long long t = i / g.nz;
    const int iy = (int)(t % g.ny);
    const int ix = (int)(t / g.ny);
    const double r[3] = {ix * g.dx, iy * g.dx, iz * g.dx};
    int b[3], lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      b[d] = min((int)(r[d] * g.inv_bw[d]), g.nb[d] - 1);
      lo[d] = g.nb[d] >= 3 ? -1 : 0;
      hi[d] = g.nb[d] >= 3 ? 1 : g.nb[d] - 1;
    }
    double sum = 0.0;
    for (int ox = lo[0]; ox <= hi[0]; ++ox) {
      const int bx = g.nb[0] >= 3 ? (b[0] + ox + g.nb[0]) % g.nb[0] : ox;
      for (int oy = lo[1]; oy <= hi[1]; ++oy) {
        const int by = g.nb[1] >= 3 ? (b[1] + oy + g.nb[1]) % g.nb[1] : oy;
        for (int oz = lo[2]; oz <= hi[2]; ++oz) {
          const int bz = g.nb[2] >= 3 ? (b[2] + oz + g.nb[2]) % g.nb[2] : oz;
          const int bin = (bx * g.nb[1] + by) * g.nb[2] + bz;
          for (int s = bin_start[bin]; s < bin_start[bin + 1]; ++s) {
            double r2 = 0.0;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              double dd = r[d] - sites[3 * s + d];
              dd -= g.L[d] * rint(dd / g.L[d]);
              r2 += dd * dd;
            }
            const double a = g.alpha * r2;
            if (a <= kPeakCut) sum += exp(-a);
          }
        }
      }
    }
    rho[i] = g.background + g.amplitude * sum;
  }
}

}  // namespace

extern "C" {

int cdft_lattice_size(int structure, int orientation, const long* shape, long* n_sites) {
  return guarded([&] {
    check_shape(shape);
    if (!n_sites) throw std::invalid_argument("n_sites is required");
    const Cell c = unit_cell(structure, orientation);
    *n_sites = (long)c.basis.size() * shape[0] * shape[1] * shape[2];
  });
}

int cdft_build_lattice(int structure, int orientation, const long* shape, double* positions, long capacity,
                       double* dimensions) {
  return guarded([&] {
    check_shape(shape);
    const Cell c = unit_cell(structure, orientation);
    const long n = (long)c.basis.size() * shape[0] * shape[1] * shape[2];
    if (!positions || capacity < n) throw std::invalid_argument("positions: room for n_sites * 3 doubles is required");
    // crystal.cpp:205-245: cells tiled x-fastest, the basis innermost
    long k = 0;
    for (long cz = 0; cz < shape[2]; ++cz)
      for (long cy = 0; cy < shape[1]; ++cy)
        for (long cx = 0; cx < shape[0]; ++cx) {
          const double off[3] = {(double)cx * c.dims[0], (double)cy * c.dims[1], (double)cz * c.dims[2]};
          for (const P3& b : c.basis) {
            for (int d = 0; d < 3; ++d) positions[3 * k + d] = b[d] + off[d];
            ++k;
          }
        }
    if (dimensions)
      for (int d = 0; d < 3; ++d) dimensions[d] = c.dims[d] * (double)shape[d];
  });
}

int cdft_lattice_export(const double* positions, long n_sites, const char* filename, int format) {
  return guarded([&] {
    if (!filename || n_sites < 0 || (n_sites > 0 && !positions))
      throw std::invalid_argument("positions, n_sites >= 0 and a file name are required");
    if (format != CDFT_EXPORT_XYZ && format != CDFT_EXPORT_CSV) throw std::invalid_argument("unknown export format");
    std::ofstream out(filename);
    if (!out) throw std::runtime_error(std::string("Cannot open file for writing: ") + filename);
    // crystal.cpp:257-279: default stream formatting (6 significant digits)
    if (format == CDFT_EXPORT_XYZ) {
      out << n_sites << "\n" << "Crystal lattice\n";
      for (long i = 0; i < n_sites; ++i)
        out << "Ar " << positions[3 * i] << " " << positions[3 * i + 1] << " " << positions[3 * i + 2] << "\n";
    } else {
      out << "x,y,z\n";
      for (long i = 0; i < n_sites; ++i)
        out << positions[3 * i] << "," << positions[3 * i + 1] << "," << positions[3 * i + 2] << "\n";
    }
    if (!out) throw std::runtime_error(std::string("write failed: ") + filename);
  });
}

int cdft_gaussian_peaks(const long* shape, double dx, const double* sites, long n_sites, double alpha,
                        double amplitude, double background, double* rho, void* stream) {
  return guarded([&] {
    if (!shape || shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0 || !(dx > 0.0))
      throw std::invalid_argument("a positive grid shape and spacing are required");
    if (!rho || n_sites < 0 || (n_sites > 0 && !sites) || !(alpha > 0.0))
      throw std::invalid_argument("rho, sites (n_sites >= 0) and alpha > 0 are required");
    if (n_sites > (1L << 30)) throw std::invalid_argument("too many sites");
    PeakGrid g;
    g.nx = (int)shape[0];
    g.ny = (int)shape[1];
    g.nz = (int)shape[2];
    g.dx = dx;
    g.alpha = alpha;
    g.amplitude = amplitude;
    g.background = background;
    const double rc = std::sqrt(kPeakCut / alpha);
    for (int d = 0; d < 3; ++d) {
      g.L[d] = (double)shape[d] * dx;
      if (g.L[d] < 2.0 * rc)
        throw std::invalid_argument("gaussian peaks: the box must be at least twice the cut radius sqrt(40/alpha)");
      g.nb[d] = (int)std::min(64.0, std::floor(g.L[d] / rc));
      g.inv_bw[d] = (double)g.nb[d] / g.L[d];
    }
    // bin the sites (wrapped into the box) by counting sort
    const int nbin = g.nb[0] * g.nb[1] * g.nb[2];
    std::vector<int> bin_of((size_t)n_sites), start((size_t)nbin + 1, 0);
    std::vector<double> w((size_t)n_sites * 3);
    for (long s = 0; s < n_sites; ++s) {
      int b[3];
      for (int d = 0; d < 3; ++d) {
        double x = std::fmod(sites[3 * s + d], g.L[d]);
        if (x < 0.0) x += g.L[d];
        if (x >= g.L[d]) x = 0.0;
        w[3 * s + d] = x;
        b[d] = std::min((int)(x * g.inv_bw[d]), g.nb[d] - 1);
      }
      bin_of[s] = (b[0] * g.nb[1] + b[1]) * g.nb[2] + b[2];
      ++start[bin_of[s] + 1];
    }
    for (int i = 0; i < nbin; ++i) start[i + 1] += start[i];
    std::vector<int> fill(start.begin(), start.end() - 1);
    std::vector<double> sorted((size_t)n_sites * 3);
    for (long s = 0; s < n_sites; ++s) {
      const int k = fill[bin_of[s]]++;
      for (int d = 0; d < 3; ++d) sorted[3 * (size_t)k + d] = w[3 * s + d];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* d_sites = nullptr;
    int* d_start = nullptr;
    CDFT_CUDA(cudaMallocAsync(&d_sites, sizeof(double) * std::max<size_t>(1, sorted.size()), st));
    CDFT_CUDA(cudaMallocAsync(&d_start, sizeof(int) * start.size(), st));
    if (!sorted.empty())
      CDFT_CUDA(cudaMemcpyAsync(d_sites, sorted.data(), sizeof(double) * sorted.size(), cudaMemcpyHostToDevice, st));
    CDFT_CUDA(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, st));
    const long long N = (long long)g.nx * g.ny * g.nz;
    const int blocks = (int)std::min<long long>((N + 255) / 256, 148LL * 16);
    k_gaussian_peaks<<<blocks, 256, 0, st>>>(g, d_sites, d_start, rho);
    const cudaError_t launch = cudaGetLastError();
    cudaFreeAsync(d_sites, st);
    cudaFreeAsync(d_start, st);
    // the host vectors above are copied from before they go out of scope
    CDFT_CUDA(cudaStreamSynchronize(st));
    CDFT_CUDA(launch);
  });
}

}  // extern "C"
