// fhd_vismf.h — one-box MultiFabs on disk in AMReX's VisMF layout (host code,
// shared by the plotfile and checkpoint writers and the checkpoint reader).
//
// <dir>/<name>_H: the VisMF header (version 1, one file, component count, ghost
// width, the BoxArray of the valid box, the FabOnDisk entry and the
// per-component minima and maxima of the written data); <dir>/<name>_D_00000:
// one FAB, a text descriptor line (little-endian IEEE doubles, the written box
// with its index type, the component count) followed by the doubles, components
// slowest and x fastest, ghost cells included.
#pragma once
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace fhd {

// creates the directory and any missing parents (as AMReX builds a plotfile's or
// checkpoint's directory hierarchy)
inline bool vismf_mkdir(const std::string& p) {
    for (size_t s = p.find('/', 1); s != std::string::npos; s = p.find('/', s + 1)) {
        const std::string part = p.substr(0, s);
        if (mkdir(part.c_str(), 0755) != 0 && errno != EEXIST) return false;
    }
    return mkdir(p.c_str(), 0755) == 0 || errno == EEXIST;
}

// AMReX's text form of a box: ((lo) (hi) (index type))
inline std::string vismf_box(const int lo[3], const int hi[3], const int type[3]) {
    char b[200];
    std::snprintf(b, sizeof(b), "((%d,%d,%d) (%d,%d,%d) (%d,%d,%d))", lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], type[0],
                  type[1], type[2]);
    return b;
}

inline const char* vismf_real_descriptor() { return "((8, (64 11 52 0 1 12 0 1023)),(8, (1 2 3 4 5 6 7 8)))"; }

// data: ncomp planes of the box glo..ghi (the valid box vlo..vhi grown by ngrow)
inline bool vismf_write(const std::string& dir, const std::string& name, const double* data, const int vlo[3],
                        const int vhi[3], const int type[3], int ncomp, int ngrow) {
    int glo[3], ghi[3];
    int64_t pts = 1;
    for (int d = 0; d < 3; ++d) {
        glo[d] = vlo[d] - ngrow;
        ghi[d] = vhi[d] + ngrow;
        pts *= (int64_t)(ghi[d] - glo[d] + 1);
    }
    FILE* f = std::fopen((dir + "/" + name + "_D_00000").c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "FAB %s%s %d\n", vismf_real_descriptor(), vismf_box(glo, ghi, type).c_str(), ncomp);
    const size_t cnt = (size_t)pts * ncomp;
    bool ok = std::fwrite(data, sizeof(double), cnt, f) == cnt;
    ok = (std::fclose(f) == 0) && ok;
    FILE* h = std::fopen((dir + "/" + name + "_H").c_str(), "w");
    if (!h) return false;
    std::fprintf(h, "1\n1\n%d\n%d\n(1 0\n%s\n)\n1\nFabOnDisk: %s_D_00000 0\n\n1,%d\n", ncomp, ngrow,
                 vismf_box(vlo, vhi, type).c_str(), name.c_str(), ncomp);
    for (int pass = 0; pass < 2; ++pass) {
        for (int c = 0; c < ncomp; ++c) {
            const double* p = data + (size_t)c * pts;
            double v = p[0];
            for (int64_t q = 1; q < pts; ++q) v = pass == 0 ? (p[q] < v ? p[q] : v) : (p[q] > v ? p[q] : v);
            std::fprintf(h, "%.17g,", v);
        }
        std::fprintf(h, pass == 0 ? "\n\n1,%d\n" : "\n", ncomp);
    }
    return (std::fclose(h) == 0) && ok;
}

// Reads <dir>/<name>_D_00000 into `out` after checking that it holds exactly the
// box glo..ghi of index type `type` with `ncomp` components: kVisOk, kVisIo (the
// file is missing, unreadable or short) or kVisShape (it holds another box).
enum { kVisOk = 0, kVisIo = 1, kVisShape = 2 };
inline int vismf_read(const std::string& dir, const std::string& name, const int glo[3], const int ghi[3],
                      const int type[3], int ncomp, std::vector<double>& out) {
    FILE* f = std::fopen((dir + "/" + name + "_D_00000").c_str(), "rb");
    if (!f) return kVisIo;
    char line[512];
    if (!std::fgets(line, sizeof(line), f)) {
        std::fclose(f);
        return kVisIo;
    }
    char want[512];
    std::snprintf(want, sizeof(want), "FAB %s%s %d\n", vismf_real_descriptor(), vismf_box(glo, ghi, type).c_str(),
                  ncomp);
    if (std::strcmp(line, want) != 0) {
        std::fclose(f);
        return kVisShape;
    }
    int64_t pts = 1;
    for (int d = 0; d < 3; ++d) pts *= (int64_t)(ghi[d] - glo[d] + 1);
    out.resize((size_t)pts * ncomp);
    const bool ok = std::fread(out.data(), sizeof(double), out.size(), f) == out.size();
    std::fclose(f);
    return ok ? kVisOk : kVisIo;
}

}  // namespace fhd
