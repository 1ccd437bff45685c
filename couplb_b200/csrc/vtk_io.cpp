// vtk_io.cpp -- VTK XML writers (see vtk_io.h).
#include "vtk_io.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace couplb {

namespace {

size_t array_bytes(const VtkArray& a) {
  return a.is_int ? a.i.size() * sizeof(int32_t) : a.f.size() * sizeof(double);
}

// <DataArray .../> header lines with appended offsets; returns the total
// appended size.
uint64_t header_arrays(FILE* fp, const std::vector<VtkArray>& arrs, uint64_t off, const char* indent) {
  for (const VtkArray& a : arrs) {
    std::fprintf(fp, "%s<DataArray type=\"%s\" Name=\"%s\"", indent, a.is_int ? "Int32" : "Float64",
                 a.name.c_str());
    if (a.ncomp > 1) std::fprintf(fp, " NumberOfComponents=\"%d\"", a.ncomp);
    std::fprintf(fp, " format=\"appended\" offset=\"%llu\"/>\n", (unsigned long long)off);
    off += sizeof(uint64_t) + array_bytes(a);
  }
  return off;
}

bool append_arrays(FILE* fp, const std::vector<VtkArray>& arrs) {
  for (const VtkArray& a : arrs) {
    const uint64_t n = array_bytes(a);
    if (std::fwrite(&n, sizeof n, 1, fp) != 1) return false;
    if (n == 0) continue;
    const void* p = a.is_int ? (const void*)a.i.data() : (const void*)a.f.data();
    if (std::fwrite(p, 1, n, fp) != n) return false;
  }
  return true;
}

}  // namespace

bool write_vti(const std::string& path, const int ext[3], const double origin[3], double spacing,
               const std::vector<VtkArray>& cells) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
  std::fprintf(fp, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" "
                   "header_type=\"UInt64\">\n");
  std::fprintf(fp, "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"%.8e %.8e %.8e\" "
                   "Spacing=\"%.8e %.8e %.8e\">\n",
               ext[0], ext[1], ext[2], origin[0], origin[1], origin[2], spacing, spacing, spacing);
  std::fprintf(fp, "    <Piece Extent=\"0 %d 0 %d 0 %d\">\n", ext[0], ext[1], ext[2]);
  std::fprintf(fp, "      <CellData Scalars=\"rho\" Vectors=\"velocity_phys\">\n");
  header_arrays(fp, cells, 0, "        ");
  std::fprintf(fp, "      </CellData>\n    </Piece>\n  </ImageData>\n");
  std::fprintf(fp, "  <AppendedData encoding=\"raw\">\n_");
  bool ok = append_arrays(fp, cells);
  std::fprintf(fp, "\n  </AppendedData>\n</VTKFile>\n");
  ok = (std::fclose(fp) == 0) && ok;
  return ok;
}

bool write_vtp(const std::string& path, const std::vector<double>& points,
               const std::vector<VtkArray>& fields) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const int np = (int)(points.size() / 3);
  std::vector<VtkArray> geo(3);
  geo[0].name = "Points";
  geo[0].ncomp = 3;
  geo[0].f = points;
  geo[1].name = "connectivity";
  geo[1].is_int = true;
  geo[2].name = "offsets";
  geo[2].is_int = true;
  geo[1].i.resize(np);
  geo[2].i.resize(np);
  for (int k = 0; k < np; k++) { geo[1].i[k] = k; geo[2].i[k] = k + 1; }
  std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
  std::fprintf(fp, "<VTKFile type=\"PolyData\" version=\"1.0\" byte_order=\"LittleEndian\" "
                   "header_type=\"UInt64\">\n");
  std::fprintf(fp, "  <PolyData>\n");
  std::fprintf(fp, "    <Piece NumberOfPoints=\"%d\" NumberOfVerts=\"%d\" NumberOfLines=\"0\" "
                   "NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n", np, np);
  uint64_t off = 0;
  std::fprintf(fp, "      <Points>\n");
  std::fprintf(fp, "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"appended\" "
                   "offset=\"%llu\"/>\n", (unsigned long long)off);
  off += sizeof(uint64_t) + array_bytes(geo[0]);
  std::fprintf(fp, "      </Points>\n      <Verts>\n");
  std::vector<VtkArray> verts(geo.begin() + 1, geo.end());
  off = header_arrays(fp, verts, off, "        ");
  std::fprintf(fp, "      </Verts>\n      <PointData>\n");
  header_arrays(fp, fields, off, "        ");
  std::fprintf(fp, "      </PointData>\n    </Piece>\n  </PolyData>\n");
  std::fprintf(fp, "  <AppendedData encoding=\"raw\">\n_");
  bool ok = append_arrays(fp, geo) && append_arrays(fp, fields);
  std::fprintf(fp, "\n  </AppendedData>\n</VTKFile>\n");
  ok = (std::fclose(fp) == 0) && ok;
  return ok;
}

bool write_pvd(const std::string& path, const std::string& prefix, const std::vector<long long>& steps,
               double dt, const char* ext) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) return false;
  std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
  std::fprintf(fp, "<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
  std::fprintf(fp, "  <Collection>\n");
  for (long long s : steps) {
    char fname[512];
    std::snprintf(fname, sizeof fname, "%s_%06lld.%s", prefix.c_str(), s, ext);
    const char* base = std::strrchr(fname, '/');
    base = base ? base + 1 : fname;
    std::fprintf(fp, "    <DataSet timestep=\"%.8e\" file=\"%s\"/>\n", (double)s * dt, base);
  }
  std::fprintf(fp, "  </Collection>\n</VTKFile>\n");
  return std::fclose(fp) == 0;
}

}  // namespace couplb
