// amrex_compat.hpp — minimal single-box stand-ins for the AMReX types that the
// reference's compressible staggered-grid interface is written against
// (amrex::MultiFab, Array4, Box, IntVect, IndexType, Geometry, Periodicity,
// Vector, Real).  They carry exactly what the reference functions read: one box
// per MultiFab, its index type (cell / face / edge), ghost width and components,
// and the domain geometry.  Memory is CUDA device memory by default; host and
// pinned host arenas exist for callers whose data lives on the host.
//
// This is not AMReX: there is no BoxArray/DistributionMapping (one box, one
// rank), no tiling, no MFIter.  Storage follows Array4 exactly (Fortran order,
// component slowest, ghost-inclusive bounds), so `fab()` hands the buffer to the
// C ABI of fhd_capi.h without a copy.
//
// Header-only C++17; needs the CUDA runtime API (link -lcudart).
#ifndef FHD_AMREX_COMPAT_HPP
#define FHD_AMREX_COMPAT_HPP

#include <cuda_runtime_api.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../fhd_capi.h"

namespace fhd {
namespace amrex_compat {

using Real = double;
template <class T>
using Vector = std::vector<T>;
template <class T, int N>
using GpuArray = std::array<T, N>;

struct IntVect {
    int v[3] = {0, 0, 0};
    IntVect() = default;
    IntVect(int a, int b, int c) : v{a, b, c} {}
    int operator[](int d) const { return v[d]; }
    int& operator[](int d) { return v[d]; }
    static IntVect TheZeroVector() { return IntVect(0, 0, 0); }
    static IntVect TheUnitVector() { return IntVect(1, 1, 1); }
    static IntVect TheDimensionVector(int d) {
        IntVect r;
        r.v[d] = 1;
        return r;
    }
    bool operator==(const IntVect& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};

// Cell- or node-centring per direction (amrex::IndexType).
struct IndexType {
    IntVect nodal;
    IndexType() = default;
    explicit IndexType(const IntVect& n) : nodal(n) {}
    bool nodeCentered(int d) const { return nodal[d] != 0; }
    bool cellCentered(int d) const { return nodal[d] == 0; }
    static IndexType TheCellType() { return IndexType(); }
    static IndexType TheNodeType() { return IndexType(IntVect(1, 1, 1)); }
};

// Inclusive index box with its centring (amrex::Box).
struct Box {
    IntVect lo, hi;
    IndexType type;
    Box() = default;
    Box(const IntVect& l, const IntVect& h, IndexType t = IndexType()) : lo(l), hi(h), type(t) {}
    const IntVect& smallEnd() const { return lo; }
    const IntVect& bigEnd() const { return hi; }
    int length(int d) const { return hi[d] - lo[d] + 1; }
    int64_t numPts() const { return int64_t(length(0)) * length(1) * length(2); }
    IndexType ixType() const { return type; }
    // amrex::convert(cc_box, nodal): the same cells, seen as the given centring
    Box convert(const IntVect& nodal) const {
        Box b = *this;
        for (int d = 0; d < 3; ++d) {
            b.hi[d] += nodal[d] - type.nodal[d];
            b.type.nodal[d] = nodal[d];
        }
        return b;
    }
    Box grow(int g) const {
        Box b = *this;
        for (int d = 0; d < 3; ++d) {
            b.lo[d] -= g;
            b.hi[d] += g;
        }
        return b;
    }
    bool operator==(const Box& o) const { return lo == o.lo && hi == o.hi && type.nodal == o.type.nodal; }
};

inline Box convert(const Box& b, const IntVect& nodal) { return b.convert(nodal); }
inline Box surroundingNodes(const Box& b, int d) {
    IntVect n = b.type.nodal;
    n[d] = 1;
    return b.convert(n);
}

struct RealBox {
    std::array<Real, 3> lo{{0, 0, 0}}, hi{{1, 1, 1}};
};

// One-box BoxArray and its (trivial) distribution, for the signatures that carry
// them (ReadCheckPoint): the box is the cell-centred domain.
struct BoxArray {
    Box box;
    void define(const Box& b) { box = b; }
};
struct DistributionMapping {};

// Every direction periodic: the only boundary the drop-in step implements.
struct Periodicity {
    IntVect period;
};

// Problem domain (amrex::Geometry): the cell-centred domain box and the
// physical extent.  All directions periodic.
struct Geometry {
    Box domain;
    RealBox prob;
    Geometry() = default;
    Geometry(const Box& dom, const RealBox& rb) : domain(dom), prob(rb) {}
    const Box& Domain() const { return domain; }
    Real CellSize(int d) const { return (prob.hi[d] - prob.lo[d]) / domain.length(d); }
    const Real* ProbLo() const { return prob.lo.data(); }
    const Real* ProbHi() const { return prob.hi.data(); }
    bool isPeriodic(int) const { return true; }
    Periodicity periodicity() const {
        return Periodicity{IntVect(domain.length(0), domain.length(1), domain.length(2))};
    }
};

// Array4 view: (i, j, k, n) with ghost-aware indices, i fastest, n slowest.
template <class T>
struct Array4 {
    T* p = nullptr;
    int64_t jstride = 0, kstride = 0, nstride = 0;
    IntVect begin, end;  // end exclusive, as in AMReX
    int ncomp = 0;
    T& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - begin[0]) + (j - begin[1]) * jstride + (k - begin[2]) * kstride + n * nstride];
    }
};

enum class Arena { Device, Pinned, Host };

[[noreturn]] inline void throw_cuda(cudaError_t e, const char* what) {
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// One box of an amrex::MultiFab, owning its memory.
class MultiFab {
  public:
    MultiFab() = default;
    // `valid` is the box of valid points (cell-centred domain box converted to
    // the wanted index type); `ngrow` ghost points on each side.
    MultiFab(const Box& valid, int ncomp, int ngrow, Arena arena = Arena::Device)
        : valid_(valid), ncomp_(ncomp), ngrow_(ngrow), arena_(arena) {
        if (ncomp < 1 || ngrow < 0) throw std::invalid_argument("MultiFab: ncomp >= 1, ngrow >= 0");
        const size_t bytes = size_t(numPtsGrown()) * size_t(ncomp) * sizeof(Real);
        cudaError_t e = cudaSuccess;
        switch (arena_) {
            case Arena::Device: e = cudaMalloc(reinterpret_cast<void**>(&data_), bytes); break;
            case Arena::Pinned: e = cudaMallocHost(reinterpret_cast<void**>(&data_), bytes); break;
            case Arena::Host:
                data_ = static_cast<Real*>(std::calloc(bytes / sizeof(Real), sizeof(Real)));
                if (!data_) throw std::bad_alloc();
                break;
        }
        if (e != cudaSuccess) {
            data_ = nullptr;
            throw_cuda(e, "MultiFab allocation");
        }
        if (arena_ == Arena::Device) {
            e = cudaMemset(data_, 0, bytes);
            if (e != cudaSuccess) throw_cuda(e, "MultiFab zero fill");
        } else if (arena_ == Arena::Pinned) {
            std::memset(data_, 0, bytes);
        }
    }
    MultiFab(const MultiFab&) = delete;
    MultiFab& operator=(const MultiFab&) = delete;
    MultiFab(MultiFab&& o) noexcept { swap(o); }
    MultiFab& operator=(MultiFab&& o) noexcept {
        if (this != &o) {
            release();
            swap(o);
        }
        return *this;
    }
    ~MultiFab() { release(); }

    // define() as in AMReX, for arrays of MultiFabs built in two steps.
    void define(const Box& valid, int ncomp, int ngrow, Arena arena = Arena::Device) {
        *this = MultiFab(valid, ncomp, ngrow, arena);
    }

    bool ok() const { return data_ != nullptr; }
    int nComp() const { return ncomp_; }
    int nGrow() const { return ngrow_; }
    IndexType ixType() const { return valid_.type; }
    const Box& validBox() const { return valid_; }
    Box grownBox() const { return valid_.grow(ngrow_); }
    Arena arena() const { return arena_; }
    int64_t numPtsGrown() const { return grownBox().numPts(); }
    int64_t size() const { return numPtsGrown() * ncomp_; }
    Real* dataPtr() const { return data_; }

    Array4<Real> array() const {
        Array4<Real> a;
        const Box g = grownBox();
        a.p = data_;
        a.jstride = g.length(0);
        a.kstride = a.jstride * g.length(1);
        a.nstride = a.kstride * g.length(2);
        a.begin = g.lo;
        a.end = IntVect(g.hi[0] + 1, g.hi[1] + 1, g.hi[2] + 1);
        a.ncomp = ncomp_;
        return a;
    }

    // The C-ABI view of this box (no copy).  An undefined MultiFab gives the
    // empty fab that optional by-product arguments take to mean "skip".
    fhd_fab fab() const {
        fhd_fab f;
        std::memset(&f, 0, sizeof(f));
        if (!data_) return f;
        const Box g = grownBox();
        f.data = data_;
        for (int d = 0; d < 3; ++d) {
            f.lo[d] = g.lo[d];
            f.hi[d] = g.hi[d];
            f.nodal[d] = valid_.type.nodal[d];
        }
        f.ncomp = ncomp_;
        f.dtype = FHD_F64;
        return f;
    }

    // Whole-buffer copies between any arenas (host vector in Array4 order).
    void copyToHost(std::vector<Real>& out) const {
        out.resize(size_t(size()));
        copy_raw(out.data(), data_, size_t(size()) * sizeof(Real));
    }
    void copyFromHost(const std::vector<Real>& in) {
        if (int64_t(in.size()) != size()) throw std::invalid_argument("copyFromHost: size mismatch");
        copy_raw(data_, in.data(), in.size() * sizeof(Real));
    }
    // MultiFab::Copy(dst, src, 0, 0, ncomp, ngrow) for same-shaped MultiFabs
    // (any arenas): every point, ghosts included.
    static void Copy(MultiFab& dst, const MultiFab& src) {
        if (!(dst.valid_ == src.valid_) || dst.ncomp_ != src.ncomp_ || dst.ngrow_ != src.ngrow_)
            throw std::invalid_argument("MultiFab::Copy: shapes differ");
        copy_raw(dst.data_, src.data_, size_t(src.size()) * sizeof(Real));
    }
    // setVal(v) on every point and component, ghosts included.
    void setVal(Real v) {
        std::vector<Real> h(size_t(size()), v);
        copyFromHost(h);
    }

    // Periodic ghost fill and nodal-duplicate sync on the device, through the
    // C ABI (device arena only).  Defined in fhd/reference_api.hpp, which owns
    // the process-wide context these run on.
    inline void FillBoundary(const Periodicity& period);
    inline void OverrideSync(const Periodicity& period);

  private:
    static void copy_raw(void* dst, const void* src, size_t bytes) {
        cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDefault);
        if (e != cudaSuccess) throw_cuda(e, "MultiFab copy");
    }
    void release() {
        if (!data_) return;
        switch (arena_) {
            case Arena::Device: cudaFree(data_); break;
            case Arena::Pinned: cudaFreeHost(data_); break;
            case Arena::Host: std::free(data_); break;
        }
        data_ = nullptr;
    }
    void swap(MultiFab& o) noexcept {
        std::swap(valid_, o.valid_);
        std::swap(ncomp_, o.ncomp_);
        std::swap(ngrow_, o.ngrow_);
        std::swap(arena_, o.arena_);
        std::swap(data_, o.data_);
    }

    Box valid_;
    int ncomp_ = 0;
    int ngrow_ = 0;
    Arena arena_ = Arena::Device;
    Real* data_ = nullptr;
};

// Nodal flags of the staggered fields (AMReX nodal IntVects).
inline IntVect face_nodal(int d) { return IntVect::TheDimensionVector(d); }
inline IntVect edge_nodal(int d1, int d2) {
    IntVect n;
    n[d1] = 1;
    n[d2] = 1;
    return n;
}

}  // namespace amrex_compat
}  // namespace fhd

#endif
