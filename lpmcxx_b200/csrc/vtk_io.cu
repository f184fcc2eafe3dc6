// Field output in the reference's file formats (host code).
//
// lpm_write_vtk writes the legacy ASCII VTK POLYDATA file that MeshedParticles::writeToVtkFile produces
// (src/LpmMeshedParticles.cpp:131-153 over VtkWriter, src/LpmVtkFileIO.cpp:12-118,195-236): header,
// POINTS, POLYGONS of the leaf faces, POINT_DATA (Lagrangian coordinates, vertex fields), CELL_DATA (face
// fields at the leaf faces).  Doubles are printed as the reference's stream prints them after
// setprecision(numeric_limits<long double>::digits10 + 1): printf's "%.19g", produced here by
// std::to_chars (general format, precision 19), which the C++ standard defines as that printf
// conversion.  lpm_write_csv writes VtkWriter::writePointsAndFieldsToCSV's layout
// (src/LpmVtkFileIO.cpp:117-193) at the stream's default precision ("%g").
//
// Coordinates and fields may live on the device: they are copied to the host (after a device-wide
// synchronize) before formatting.  Formatting is split over host threads in contiguous row ranges and
// written in order.
#include "lpm_internal.h"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace lpm {
namespace {

constexpr int kVtkPrecision = 19;  // numeric_limits<long double>::digits10 + 1 on x86-64
constexpr int kCsvPrecision = 6;   // a fresh stream's default precision

inline void put_double(std::string& s, double v, int prec) {
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, prec);
    s.append(buf, r.ptr);
}

inline void put_int(std::string& s, int64_t v) {
    char buf[24];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v);
    s.append(buf, r.ptr);
}

// Rows [0, n) formatted by fn(row, string&) on up to 16 host threads, appended to out in row order.
template <class Fn>
void format_rows(int64_t n, std::string& out, Fn fn) {
    const int64_t per = 16384;
    const int hw = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int nt = (int)std::min<int64_t>(hw, (n + per - 1) / per);
    if (nt <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i, out);
        return;
    }
    std::vector<std::string> parts(nt);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            const int64_t i0 = n * t / nt, i1 = n * (t + 1) / nt;
            parts[t].reserve((size_t)(i1 - i0) * 64);
            for (int64_t i = i0; i < i1; ++i) fn(i, parts[t]);
        });
    for (auto& x : th) x.join();
    for (auto& p : parts) out += p;
}

// Host copy of n items of `cols` doubles with the given stride (in doubles) or component-major layout.
struct HostArray {
    std::vector<double> own;
    const double* p = nullptr;
};

int fetch(const double* data, size_t count, bool on_device, HostArray& h) {
    if (!on_device) {
        h.p = data;
        return LPM_OK;
    }
    h.own.resize(count);
    if (count) {
        LPM_CUDA_TRY(cudaDeviceSynchronize());
        LPM_CUDA_TRY(cudaMemcpy(h.own.data(), data, count * sizeof(double), cudaMemcpyDeviceToHost));
    }
    h.p = h.own.data();
    return LPM_OK;
}

int check_fields(int32_t nf, const lpm_field_desc* f, const char* where) {
    if (nf < 0 || (nf > 0 && !f)) {
        set_error("%s: bad field list", where);
        return LPM_ERR_ARG;
    }
    for (int32_t k = 0; k < nf; ++k)
        if (!f[k].name || !f[k].units || f[k].ndim < 1 || f[k].ndim > 3 || !f[k].data) {
            set_error("%s: field %d needs a name, units, 1 <= ndim <= 3 and data", where, (int)k);
            return LPM_ERR_ARG;
        }
    return LPM_OK;
}

bool write_file(const char* path, const std::string& s) {
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    return std::fclose(fp) == 0 && ok;
}

// "SCALARS <name>_<units> double <ndim>\nLOOKUP_TABLE default\n" and the values of the selected items
// (src/LpmVtkFileIO.cpp:74-103, 195-236).
int vtk_field(std::string& s, const lpm_field_desc& f, int64_t n, const std::vector<int64_t>* rows) {
    HostArray h;
    int rc = fetch(f.data, (size_t)f.ndim * (size_t)n, f.on_device != 0, h);
    if (rc) return rc;
    s += "SCALARS ";
    s += f.name;
    s += "_";
    s += f.units;
    s += " double ";
    put_int(s, f.ndim);
    s += "\nLOOKUP_TABLE default\n";
    const int64_t m = rows ? (int64_t)rows->size() : n;
    const double* d = h.p;
    const int nd = f.ndim;
    format_rows(m, s, [&](int64_t r, std::string& o) {
        const int64_t i = rows ? (*rows)[r] : r;
        for (int c = 0; c < nd; ++c) {
            if (c) o += ' ';
            put_double(o, d[(size_t)c * n + i], kVtkPrecision);
        }
        o += '\n';
    });
    return LPM_OK;
}

}  // namespace
}  // namespace lpm

using namespace lpm;

extern "C" int lpm_write_vtk(const char* path, const char* title, int64_t n_verts, const double* vert_xyz,
                             int32_t xyz_stride, int32_t xyz_on_device, const double* lag_xyz, int64_t n_faces,
                             int32_t nsides, const int64_t* face_verts, const uint8_t* face_divided,
                             int32_t n_vert_fields, const lpm_field_desc* vert_fields, int32_t n_face_fields,
                             const lpm_field_desc* face_fields) {
    if (!path || n_verts < 0 || n_faces < 0 || (n_verts > 0 && !vert_xyz) || xyz_stride < 3 || nsides < 3 ||
        (n_faces > 0 && (!face_verts || !face_divided))) {
        set_error("lpm_write_vtk: bad arguments");
        return LPM_ERR_ARG;
    }
    int rc = check_fields(n_vert_fields, vert_fields, "lpm_write_vtk");
    if (!rc) rc = check_fields(n_face_fields, face_fields, "lpm_write_vtk");
    if (rc) return rc;
    std::vector<int64_t> leaves;
    for (int64_t f = 0; f < n_faces; ++f) {
        if (face_divided[f]) continue;
        for (int j = 0; j < nsides; ++j) {
            const int64_t v = face_verts[f * nsides + j];
            if (v < 0 || v >= n_verts) {
                set_error("lpm_write_vtk: face %lld names vertex %lld of %lld", (long long)f, (long long)v,
                          (long long)n_verts);
                return LPM_ERR_ARG;
            }
        }
        leaves.push_back(f);
    }
    const size_t xyz_count = n_verts > 0 ? (size_t)(n_verts - 1) * xyz_stride + 3 : 0;
    HostArray X, Lg;
    rc = fetch(vert_xyz, xyz_count, xyz_on_device != 0, X);
    if (!rc && lag_xyz) rc = fetch(lag_xyz, xyz_count, xyz_on_device != 0, Lg);
    if (rc) return rc;
    std::string s;
    try {
        s.reserve((size_t)n_verts * 80 + leaves.size() * 40);
        // header and points (src/LpmVtkFileIO.cpp:12-26)
        s += "# vtk DataFile Version 2.0\n";
        s += title ? title : "";
        s += "\nASCII\nDATASET POLYDATA\nPOINTS ";
        put_int(s, n_verts);
        s += " double\n";
        auto coords = [&](const double* p) {
            format_rows(n_verts, s, [&](int64_t i, std::string& o) {
                const double* q = p + (size_t)i * xyz_stride;
                put_double(o, q[0], kVtkPrecision);
                o += ' ';
                put_double(o, q[1], kVtkPrecision);
                o += ' ';
                put_double(o, q[2], kVtkPrecision);
                o += '\n';
            });
        };
        coords(X.p);
        // leaf polygons, each index followed by a space (src/LpmVtkFileIO.cpp:28-53)
        s += "POLYGONS ";
        put_int(s, (int64_t)leaves.size());
        s += ' ';
        put_int(s, (int64_t)leaves.size() * (nsides + 1));
        s += '\n';
        format_rows((int64_t)leaves.size(), s, [&](int64_t r, std::string& o) {
            put_int(o, nsides);
            o += ' ';
            for (int j = 0; j < nsides; ++j) {
                put_int(o, face_verts[leaves[r] * nsides + j]);
                o += ' ';
            }
            o += '\n';
        });
        // point data (src/LpmVtkFileIO.cpp:55-72; src/LpmMeshedParticles.cpp:142-147)
        s += "POINT_DATA ";
        put_int(s, n_verts);
        s += '\n';
        if (lag_xyz) {
            s += "SCALARS lagrangian_coords double 3\nLOOKUP_TABLE default\n";
            coords(Lg.p);
        }
        for (int32_t k = 0; k < n_vert_fields; ++k)
            if ((rc = vtk_field(s, vert_fields[k], n_verts, nullptr))) return rc;
        // cell data at the leaf faces (src/LpmVtkFileIO.cpp:105-107,195-236)
        s += "CELL_DATA ";
        put_int(s, (int64_t)leaves.size());
        s += '\n';
        for (int32_t k = 0; k < n_face_fields; ++k)
            if ((rc = vtk_field(s, face_fields[k], n_faces, &leaves))) return rc;
    } catch (const std::bad_alloc&) {
        set_error("lpm_write_vtk: out of host memory");
        return LPM_ERR_OOM;
    }
    if (!write_file(path, s)) {
        set_error("lpm_write_vtk: cannot write %s", path);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

extern "C" int lpm_write_csv(const char* path, int64_t n, const double* xyz, int32_t xyz_stride,
                             int32_t xyz_on_device, int32_t n_fields, const lpm_field_desc* fields) {
    if (!path || n < 0 || (n > 0 && !xyz) || xyz_stride < 3) {
        set_error("lpm_write_csv: bad arguments");
        return LPM_ERR_ARG;
    }
    int rc = check_fields(n_fields, fields, "lpm_write_csv");
    if (rc) return rc;
    HostArray X;
    rc = fetch(xyz, n > 0 ? (size_t)(n - 1) * xyz_stride + 3 : 0, xyz_on_device != 0, X);
    if (rc) return rc;
    std::vector<HostArray> F(n_fields);
    for (int32_t k = 0; k < n_fields; ++k)
        if ((rc = fetch(fields[k].data, (size_t)fields[k].ndim * (size_t)n, fields[k].on_device != 0, F[k])))
            return rc;
    std::string s;
    try {
        // header: x,y,z then name or name0,name1[,name2] per field (src/LpmVtkFileIO.cpp:119-157)
        s += "x,y,z";
        for (int32_t k = 0; k < n_fields; ++k) {
            if (fields[k].ndim == 1) {
                s += ',';
                s += fields[k].name;
            } else {
                for (int c = 0; c < fields[k].ndim; ++c) {
                    s += ',';
                    s += fields[k].name;
                    put_int(s, c);
                }
            }
        }
        s += '\n';
        format_rows(n, s, [&](int64_t i, std::string& o) {
            const double* q = X.p + (size_t)i * xyz_stride;
            for (int c = 0; c < 3; ++c) {
                if (c) o += ',';
                put_double(o, q[c], kCsvPrecision);
            }
            for (int32_t k = 0; k < n_fields; ++k)
                for (int c = 0; c < fields[k].ndim; ++c) {
                    o += ',';
                    put_double(o, F[k].p[(size_t)c * n + i], kCsvPrecision);
                }
            o += '\n';
        });
    } catch (const std::bad_alloc&) {
        set_error("lpm_write_csv: out of host memory");
        return LPM_ERR_OOM;
    }
    if (!write_file(path, s)) {
        set_error("lpm_write_csv: cannot write %s", path);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}
