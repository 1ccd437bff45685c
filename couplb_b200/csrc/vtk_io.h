// vtk_io.h -- VTK XML writers of the fix's field and solid output (host).
// Same files, names and layout as the reference's IO::write_vtk /
// write_solid_vtk / write_pvd (couplb_io.h:42-306, 309-614), but with the
// arrays as raw little-endian binary in an AppendedData block (UInt64 length
// headers) instead of ASCII text.  Not part of the public ABI.
#pragma once
#include <string>
#include <vector>

namespace couplb {

// One array of a VTK file: ncomp components per tuple.
struct VtkArray {
  std::string name;
  int ncomp = 1;
  bool is_int = false;                 // Int32, else Float64
  std::vector<double> f;               // tuples x ncomp (Float64)
  std::vector<int> i;                  // tuples x ncomp (Int32)
};

// ImageData of Rx x Ry x Rz cells (cell data), origin / spacing in MD units.
bool write_vti(const std::string& path, const int ext[3], const double origin[3], double spacing,
               const std::vector<VtkArray>& cells);

// PolyData of npts vertices (point data).
bool write_vtp(const std::string& path, const std::vector<double>& points,
               const std::vector<VtkArray>& fields);

// Collection listing <prefix>_<step %06ld>.<ext> at time step * dt.
bool write_pvd(const std::string& path, const std::string& prefix, const std::vector<long long>& steps,
               double dt, const char* ext);

}  // namespace couplb
