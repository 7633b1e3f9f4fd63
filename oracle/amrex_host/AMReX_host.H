// AMReX_host.H — a serial, host-only, single-box stand-in for the part of the
// AMReX API that FHDeX's compressible staggered path uses, written here so
// that the reference's own hot-path sources (timeStepStag.cpp, fluxStag.cpp,
// conservedPrimitiveConversionsStag.cpp, transCoeffs.cpp, ...) compile
// UNMODIFIED into a CPU library (oracle/_ref) that pins the restated oracle.
// Test infrastructure only: nothing in the product links it.
//
// Semantics restated (AMReX itself is not available here):
//  * one box per MultiFab (BoxArray of one box, one "rank"); MFIter makes one
//    tile equal to the valid box, so tilebox() == validbox() and the nodal /
//    grown variants derive from it; ParallelFor runs serial loops, i fastest;
//  * Array4 / FArrayBox in Fortran order with the component slowest, storage
//    over the box grown by nGrow (ghost cells);
//  * MultiFab::LinComb dst = a*x + b*y, Copy, setVal, mult, plus;
//  * FillBoundary(periodicity): every ghost point outside the valid box (cell
//    or nodal) takes the value of its periodic image inside the valid box;
//  * OverrideSync(periodicity) on nodal data: a point on the high boundary of a
//    periodic nodal direction takes the value of its image on the low boundary
//    (the low-side point is the owner);
//  * FillRandomNormal / ParallelForRNG + RandomNormal do not draw: they take
//    their standard normals from a caller-installed source (injected noise),
//    and return mean + stddev * z as a normal draw would;
//  * ParmParse reads "key = values" lines from an in-memory table;
//  * ParallelDescriptor is a single process;
//  * sumToLine(mf, icomp, ncomp, domain, dir, local) returns, for every index m
//    along dir and component n, the sum of mf over the valid box's plane at m in
//    the host vector's entry m*ncomp + n (the layout the reference indexes),
//    accumulated from 0.0 in the box's loop order (z slowest, x fastest), so
//    that for the x line each entry sums its plane with k outer and j inner.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <numeric>
#include <sstream>
#include <limits>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#define AMREX_SPACEDIM 3
#define BL_SPACEDIM 3
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_PICK(a, b, c) c
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_MANAGED
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
#define AMREX_ASSERT(x) ((void)0)
#define AMREX_ALWAYS_ASSERT(x) do { if (!(x)) amrex::Abort("assertion failed: " #x); } while (0)
#define BL_ASSERT(x) ((void)0)
#define BL_PROFILE(a)
#define BL_PROFILE_VAR(a, b)
#define BL_PROFILE_VAR_NS(a, b)
#define BL_PROFILE_VAR_START(a)
#define BL_PROFILE_VAR_STOP(a)
#define AMREX_GPU_ERROR_CHECK()

namespace amrex {

using Real = double;
using Long = long long;

// Abort: the reference's physics guards end here; the harness installs a
// handler that unwinds (throws) so that the test sees the failure.
using AbortHandler = void (*)(const char*);
inline AbortHandler& abort_handler() {
    static AbortHandler h = nullptr;
    return h;
}
[[noreturn]] inline void Abort(const char* msg = "") {
    if (abort_handler()) abort_handler()(msg);
    std::fprintf(stderr, "amrex::Abort: %s\n", msg);
    std::abort();
}
[[noreturn]] inline void Abort(const std::string& msg) { Abort(msg.c_str()); }
inline void Warning(const std::string& msg) { std::fprintf(stderr, "amrex::Warning: %s\n", msg.c_str()); }

// Print(): a quiet stream (the reference's diagnostics are not part of the result)
struct Print {
    std::ostringstream os;
    Print() = default;
    explicit Print(int) {}
    explicit Print(std::ostream&) {}
    template <class T>
    Print& operator<<(const T& v) { os << v; return *this; }
    Print& operator<<(std::ostream& (*f)(std::ostream&)) { os << f; return *this; }
    Print& SetPrecision(int p) { os.precision(p); return *this; }
};
using AllPrint = Print;

template <class T>
class Vector : public std::vector<T> {
public:
    using std::vector<T>::vector;
    T* dataPtr() { return this->data(); }
    const T* dataPtr() const { return this->data(); }
};

template <class T, int N>
struct GpuArray {
    T arr[N];
    T& operator[](int i) { return arr[i]; }
    const T& operator[](int i) const { return arr[i]; }
    T* data() { return arr; }
    const T* data() const { return arr; }
    static constexpr int size() { return N; }
    T* begin() { return arr; }
    T* end() { return arr + N; }
};
template <class T, size_t N>
using Array = std::array<T, N>;

enum class Order { C, F };
// Array2D<T, XLO, XHI, YLO, YHI>: both bounds inclusive
template <class T, int XLO, int XHI, int YLO, int YHI, Order ORDER = Order::F>
struct Array2D {
    T arr[(XHI - XLO + 1) * (YHI - YLO + 1)];
    T& operator()(int i, int j) { return arr[(i - XLO) + (j - YLO) * (XHI - XLO + 1)]; }
    const T& operator()(int i, int j) const { return arr[(i - XLO) + (j - YLO) * (XHI - XLO + 1)]; }
};

namespace Math {
template <class T> inline T abs(T x) { return std::abs(x); }
template <int P, class T> inline T powi(T x) { T r = 1; for (int q = 0; q < P; ++q) r *= x; return r; }
inline double pi() { return 3.14159265358979323846; }
template <class T> inline T floor(T x) { return std::floor(x); }
}  // namespace Math
template <class T> inline const T& min(const T& a, const T& b) { return std::min(a, b); }
template <class T> inline const T& max(const T& a, const T& b) { return std::max(a, b); }
template <class T, class... R> inline T min(const T& a, const T& b, const R&... r) { return min(min(a, b), r...); }
template <class T, class... R> inline T max(const T& a, const T& b, const R&... r) { return max(max(a, b), r...); }
template <class T> inline T Clamp(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }
using std::get;

namespace Gpu {
template <class T> using HostVector = Vector<T>;
template <class T> using DeviceVector = Vector<T>;
template <class T> using ManagedVector = Vector<T>;
struct HostToDevice {};
struct DeviceToHost {};
struct DeviceToDevice {};
constexpr HostToDevice hostToDevice{};
constexpr DeviceToHost deviceToHost{};
constexpr DeviceToDevice deviceToDevice{};
template <class Tag, class It, class Out> void copy(Tag, It b, It e, Out o) { std::copy(b, e, o); }
template <class Tag, class It, class Out> void copyAsync(Tag, It b, It e, Out o) { std::copy(b, e, o); }
inline void synchronize() {}
inline void streamSynchronize() {}
struct Device { static void synchronize() {} static void streamSynchronize() {} };
inline bool inLaunchRegion() { return false; }
inline bool notInLaunchRegion() { return true; }
}  // namespace Gpu

// ---- index space -----------------------------------------------------------------
struct Dim3 { int x, y, z; };

class IntVect {
public:
    int vect[3];
    IntVect() : vect{0, 0, 0} {}
    IntVect(int i, int j, int k) : vect{i, j, k} {}
    explicit IntVect(int v) : vect{v, v, v} {}
    explicit IntVect(const int* v) : vect{v[0], v[1], v[2]} {}
    explicit IntVect(const std::vector<int>& v) : vect{v[0], v[1], v[2]} {}
    int& operator[](int d) { return vect[d]; }
    const int& operator[](int d) const { return vect[d]; }
    bool operator==(const IntVect& o) const { return vect[0] == o[0] && vect[1] == o[1] && vect[2] == o[2]; }
    bool operator!=(const IntVect& o) const { return !(*this == o); }
    IntVect operator+(const IntVect& o) const { return {vect[0] + o[0], vect[1] + o[1], vect[2] + o[2]}; }
    IntVect operator-(const IntVect& o) const { return {vect[0] - o[0], vect[1] - o[1], vect[2] - o[2]}; }
    IntVect operator-() const { return {-vect[0], -vect[1], -vect[2]}; }
    IntVect operator*(int s) const { return {vect[0] * s, vect[1] * s, vect[2] * s}; }
    IntVect& operator+=(const IntVect& o) { for (int d = 0; d < 3; ++d) vect[d] += o[d]; return *this; }
    IntVect& operator-=(const IntVect& o) { for (int d = 0; d < 3; ++d) vect[d] -= o[d]; return *this; }
    int max() const { return std::max(vect[0], std::max(vect[1], vect[2])); }
    int min() const { return std::min(vect[0], std::min(vect[1], vect[2])); }
    bool allGE(const IntVect& o) const { return vect[0] >= o[0] && vect[1] >= o[1] && vect[2] >= o[2]; }
    bool allLE(const IntVect& o) const { return vect[0] <= o[0] && vect[1] <= o[1] && vect[2] <= o[2]; }
    Dim3 dim3() const { return {vect[0], vect[1], vect[2]}; }
    const int* getVect() const { return vect; }
    static IntVect TheZeroVector() { return IntVect(0); }
    static IntVect TheUnitVector() { return IntVect(1); }
    static IntVect TheNodeVector() { return IntVect(1); }
    static IntVect TheCellVector() { return IntVect(0); }
};
inline std::ostream& operator<<(std::ostream& os, const IntVect& v) {
    return os << "(" << v[0] << "," << v[1] << "," << v[2] << ")";
}

class IndexType {
public:
    IntVect t;  // 1 = nodal in that direction
    IndexType() = default;
    explicit IndexType(const IntVect& v) : t(v) {}
    bool nodeCentered(int d) const { return t[d] == 1; }
    bool cellCentered(int d) const { return t[d] == 0; }
    bool nodeCentered() const { return t == IntVect(1); }
    bool cellCentered() const { return t == IntVect(0); }
    IntVect toIntVect() const { return t; }
    IntVect ixType() const { return t; }
    int operator[](int d) const { return t[d]; }
    bool operator==(const IndexType& o) const { return t == o.t; }
    bool operator!=(const IndexType& o) const { return t != o.t; }
    static IndexType TheCellType() { return IndexType(IntVect(0)); }
    static IndexType TheNodeType() { return IndexType(IntVect(1)); }
};

class Orientation {
public:
    enum Side { low = 0, high = 1 };
    int dir_, side_;
    Orientation(int dir, Side s) : dir_(dir), side_(s) {}
    int coordDir() const { return dir_; }
    bool isLow() const { return side_ == low; }
    bool isHigh() const { return side_ == high; }
};

class Box {
public:
    IntVect lo, hi;
    IndexType typ;
    Box() : lo(0), hi(-1) {}
    Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
    Box(const IntVect& l, const IntVect& h, const IntVect& type) : lo(l), hi(h), typ(type) {}
    Box(const IntVect& l, const IntVect& h, const IndexType& type) : lo(l), hi(h), typ(type) {}
    const IntVect& smallEnd() const { return lo; }
    const IntVect& bigEnd() const { return hi; }
    int smallEnd(int d) const { return lo[d]; }
    int bigEnd(int d) const { return hi[d]; }
    const int* loVect() const { return lo.vect; }
    const int* hiVect() const { return hi.vect; }
    IntVect size() const { return hi - lo + IntVect(1); }
    IntVect length() const { return size(); }
    int length(int d) const { return hi[d] - lo[d] + 1; }
    Long numPts() const {
        if (!ok()) return 0;
        return (Long)length(0) * length(1) * length(2);
    }
    bool ok() const { return hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]; }
    bool isEmpty() const { return !ok(); }
    IndexType ixType() const { return typ; }
    IntVect type() const { return typ.t; }
    int type(int d) const { return typ.t[d]; }
    bool contains(const IntVect& p) const { return p.allGE(lo) && p.allLE(hi); }
    bool contains(const Box& b) const { return b.lo.allGE(lo) && b.hi.allLE(hi); }
    bool intersects(const Box& b) const {
        for (int d = 0; d < 3; ++d)
            if (std::max(lo[d], b.lo[d]) > std::min(hi[d], b.hi[d])) return false;
        return true;
    }
    Box& setSmall(int d, int v) { lo[d] = v; return *this; }
    Box& setBig(int d, int v) { hi[d] = v; return *this; }
    Box& setSmall(const IntVect& v) { lo = v; return *this; }
    Box& setBig(const IntVect& v) { hi = v; return *this; }
    Box& grow(int n) { lo -= IntVect(n); hi += IntVect(n); return *this; }
    Box& grow(const IntVect& n) { lo -= n; hi += n; return *this; }
    Box& grow(int d, int n) { lo[d] -= n; hi[d] += n; return *this; }
    Box& growLo(int d, int n = 1) { lo[d] -= n; return *this; }
    Box& growHi(int d, int n = 1) { hi[d] += n; return *this; }
    Box& shift(int d, int n) { lo[d] += n; hi[d] += n; return *this; }
    Box& shift(const IntVect& v) { lo += v; hi += v; return *this; }
    // index-type changes keep the cells they cover: cell -> node adds the high node
    Box& surroundingNodes() { for (int d = 0; d < 3; ++d) surroundingNodes(d); return *this; }
    Box& surroundingNodes(int d) {
        if (typ.t[d] == 0) { typ.t[d] = 1; hi[d] += 1; }
        return *this;
    }
    Box& enclosedCells() { for (int d = 0; d < 3; ++d) enclosedCells(d); return *this; }
    Box& enclosedCells(int d) {
        if (typ.t[d] == 1) { typ.t[d] = 0; hi[d] -= 1; }
        return *this;
    }
    Box& convert(const IntVect& t) {
        for (int d = 0; d < 3; ++d) {
            if (t[d] == 1) surroundingNodes(d);
            else enclosedCells(d);
        }
        return *this;
    }
    Box& convert(const IndexType& t) { return convert(t.t); }
    Box& makeSlab(int d, int v) { lo[d] = v; hi[d] = v; return *this; }
    Box operator&(const Box& b) const {
        Box r(*this);
        for (int d = 0; d < 3; ++d) { r.lo[d] = std::max(lo[d], b.lo[d]); r.hi[d] = std::min(hi[d], b.hi[d]); }
        return r;
    }
    Box& operator&=(const Box& b) { *this = *this & b; return *this; }
    bool operator==(const Box& b) const { return lo == b.lo && hi == b.hi && typ == b.typ; }
    bool operator!=(const Box& b) const { return !(*this == b); }
};
inline Box grow(const Box& b, int n) { Box r(b); return r.grow(n); }
inline Box grow(const Box& b, const IntVect& n) { Box r(b); return r.grow(n); }
inline Box grow(const Box& b, int d, int n) { Box r(b); return r.grow(d, n); }
inline Box growLo(const Box& b, int d, int n) { Box r(b); return r.growLo(d, n); }
inline Box growHi(const Box& b, int d, int n) { Box r(b); return r.growHi(d, n); }
inline Box convert(const Box& b, const IntVect& t) { Box r(b); return r.convert(t); }
inline Box convert(const Box& b, const IndexType& t) { Box r(b); return r.convert(t); }
inline Box surroundingNodes(const Box& b) { Box r(b); return r.surroundingNodes(); }
inline Box surroundingNodes(const Box& b, int d) { Box r(b); return r.surroundingNodes(d); }
inline Box enclosedCells(const Box& b) { Box r(b); return r.enclosedCells(); }
inline Box shift(const Box& b, int d, int n) { Box r(b); return r.shift(d, n); }
// the nodes on one face of b (b converted to nodal in the face's direction)
inline Box bdryNode(const Box& b, Orientation face, int len = 1) {
    const int d = face.coordDir();
    Box r(b);
    r.surroundingNodes(d);
    if (face.isLow()) { r.hi[d] = r.lo[d] + len - 1; }
    else { r.lo[d] = r.hi[d] - len + 1; }
    return r;
}
inline Box bdryLo(const Box& b, int d, int len = 1) { return bdryNode(b, Orientation(d, Orientation::low), len); }
inline Box bdryHi(const Box& b, int d, int len = 1) { return bdryNode(b, Orientation(d, Orientation::high), len); }
inline Dim3 lbound(const Box& b) { return b.lo.dim3(); }
inline Dim3 ubound(const Box& b) { return b.hi.dim3(); }
inline Dim3 length(const Box& b) { return b.size().dim3(); }

class BoxArray {
public:
    std::vector<Box> boxes;
    BoxArray() = default;
    explicit BoxArray(const Box& b) : boxes{b} {}
    BoxArray(const Box* b, size_t n) : boxes(b, b + n) {}
    void define(const Box& b) { boxes = {b}; }
    int size() const { return (int)boxes.size(); }
    const Box& operator[](int i) const { return boxes[i]; }
    Box get(int i) const { return boxes[i]; }
    BoxArray& maxSize(int) { return *this; }             // one box: never split
    BoxArray& maxSize(const IntVect&) { return *this; }
    BoxArray& convert(const IntVect& t) { for (auto& b : boxes) b.convert(t); return *this; }
    BoxArray& convert(const IndexType& t) { return convert(t.t); }
    IndexType ixType() const { return boxes.empty() ? IndexType() : boxes[0].typ; }
    Box minimalBox() const { return boxes.empty() ? Box() : boxes[0]; }
    bool operator==(const BoxArray& o) const { return boxes == o.boxes; }
};
inline BoxArray convert(const BoxArray& ba, const IntVect& t) { BoxArray r(ba); return r.convert(t); }

class DistributionMapping {
public:
    DistributionMapping() = default;
    explicit DistributionMapping(const BoxArray&, int = 1) {}
    explicit DistributionMapping(std::vector<int>&&) {}
    int operator[](int) const { return 0; }
};

class RealBox {
public:
    Real xlo[3], xhi[3];
    RealBox() : xlo{0, 0, 0}, xhi{1, 1, 1} {}
    RealBox(const Real* lo, const Real* hi) { for (int d = 0; d < 3; ++d) { xlo[d] = lo[d]; xhi[d] = hi[d]; } }
    RealBox(const std::array<Real, 3>& lo, const std::array<Real, 3>& hi) {
        for (int d = 0; d < 3; ++d) { xlo[d] = lo[d]; xhi[d] = hi[d]; }
    }
    const Real* lo() const { return xlo; }
    const Real* hi() const { return xhi; }
    Real lo(int d) const { return xlo[d]; }
    Real hi(int d) const { return xhi[d]; }
    Real length(int d) const { return xhi[d] - xlo[d]; }
};

class Periodicity {
public:
    IntVect period;  // 0 = not periodic in that direction
    Periodicity() = default;
    explicit Periodicity(const IntVect& p) : period(p) {}
    bool isPeriodic(int d) const { return period[d] != 0; }
    bool isAnyPeriodic() const { return period[0] || period[1] || period[2]; }
    static Periodicity NonPeriodic() { return Periodicity(); }
};

class Geometry {
public:
    Box domain;
    RealBox prob;
    int coord = 0;
    int periodic[3] = {0, 0, 0};
    Real dx[3] = {1, 1, 1}, inv_dx[3] = {1, 1, 1};
    Geometry() = default;
    Geometry(const Box& dom, const RealBox& rb, int c, const Array<int, 3>& is_per) { define(dom, rb, c, is_per); }
    Geometry(const Box& dom, const RealBox* rb, int c, const int* is_per) {
        Array<int, 3> p{is_per[0], is_per[1], is_per[2]};
        define(dom, *rb, c, p);
    }
    void define(const Box& dom, const RealBox* rb, int c, const int* is_per) {
        Array<int, 3> p{is_per[0], is_per[1], is_per[2]};
        define(dom, *rb, c, p);
    }
    void define(const Box& dom, const RealBox& rb, int c, const Array<int, 3>& is_per) {
        domain = dom;
        prob = rb;
        coord = c;
        for (int d = 0; d < 3; ++d) {
            periodic[d] = is_per[d];
            dx[d] = (prob.hi(d) - prob.lo(d)) / domain.length(d);
            inv_dx[d] = 1.0 / dx[d];
        }
    }
    const Box& Domain() const { return domain; }
    const RealBox& ProbDomain() const { return prob; }
    const Real* CellSize() const { return dx; }
    Real CellSize(int d) const { return dx[d]; }
    GpuArray<Real, 3> CellSizeArray() const { return {{dx[0], dx[1], dx[2]}}; }
    GpuArray<Real, 3> InvCellSizeArray() const { return {{inv_dx[0], inv_dx[1], inv_dx[2]}}; }
    const Real* ProbLo() const { return prob.xlo; }
    const Real* ProbHi() const { return prob.xhi; }
    Real ProbLo(int d) const { return prob.lo(d); }
    Real ProbHi(int d) const { return prob.hi(d); }
    Real ProbLength(int d) const { return prob.length(d); }
    GpuArray<Real, 3> ProbLoArray() const { return {{prob.xlo[0], prob.xlo[1], prob.xlo[2]}}; }
    GpuArray<Real, 3> ProbHiArray() const { return {{prob.xhi[0], prob.xhi[1], prob.xhi[2]}}; }
    bool isPeriodic(int d) const { return periodic[d] != 0; }
    bool isAllPeriodic() const { return periodic[0] && periodic[1] && periodic[2]; }
    bool isAnyPeriodic() const { return periodic[0] || periodic[1] || periodic[2]; }
    Periodicity periodicity() const {
        IntVect p;
        for (int d = 0; d < 3; ++d) p[d] = periodic[d] ? domain.length(d) : 0;
        return Periodicity(p);
    }
};

// ---- data ---------------------------------------------------------------------------
template <class T>
struct Array4 {
    T* p = nullptr;
    Long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{0, 0, 0}, end{0, 0, 0};  // end exclusive
    int ncomp = 0;
    Array4() = default;
    Array4(T* ptr, Dim3 lo, Dim3 hi_excl, int nc)
        : p(ptr), jstride(hi_excl.x - lo.x), kstride((Long)(hi_excl.x - lo.x) * (hi_excl.y - lo.y)),
          nstride(kstride * (hi_excl.z - lo.z)), begin(lo), end(hi_excl), ncomp(nc) {}
    template <class U, class = typename std::enable_if<std::is_same<const U, T>::value>::type>
    Array4(const Array4<U>& o)
        : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride), begin(o.begin), end(o.end),
          ncomp(o.ncomp) {}
    T& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
    T& operator()(const IntVect& v, int n = 0) const { return (*this)(v[0], v[1], v[2], n); }
    T* ptr(int i, int j, int k, int n = 0) const { return &(*this)(i, j, k, n); }
    T* dataPtr() const { return p; }
    int nComp() const { return ncomp; }
    bool contains(int i, int j, int k) const {
        return i >= begin.x && i < end.x && j >= begin.y && j < end.y && k >= begin.z && k < end.z;
    }
    explicit operator bool() const { return p != nullptr; }
};

class FArrayBox {
public:
    Box bx;  // the box of the storage (valid box grown by the ghost width)
    int nc = 0;
    Real* dptr = nullptr;
    std::vector<Real> own;
    FArrayBox() = default;
    FArrayBox(const Box& b, int ncomp) { resize(b, ncomp); }
    FArrayBox(const Box& b, int ncomp, Real* p) { wrap(p, b, ncomp); }
    void resize(const Box& b, int ncomp) {
        bx = b;
        nc = ncomp;
        own.assign((size_t)b.numPts() * ncomp, 0.0);
        dptr = own.data();
    }
    void wrap(Real* p, const Box& b, int ncomp) { bx = b; nc = ncomp; dptr = p; own.clear(); }
    const Box& box() const { return bx; }
    int nComp() const { return nc; }
    Real* dataPtr(int n = 0) { return dptr + (size_t)n * bx.numPts(); }
    const Real* dataPtr(int n = 0) const { return dptr + (size_t)n * bx.numPts(); }
    Array4<Real> array() {
        return Array4<Real>(dptr, bx.lo.dim3(), (bx.hi + IntVect(1)).dim3(), nc);
    }
    Array4<Real const> array() const {
        return Array4<Real const>(dptr, bx.lo.dim3(), (bx.hi + IntVect(1)).dim3(), nc);
    }
    Array4<Real const> const_array() const { return array(); }
    void setVal(Real v) { std::fill(dptr, dptr + (size_t)bx.numPts() * nc, v); }
};

class MultiFab;

// Standard normals for the noise fills come from an installed source: the
// harness injects the values the reference's RNG would have drawn.
struct NoiseSource {
    // one FillRandomNormal call: write mean + stddev * z into comps scomp..scomp+ncomp-1 of mf
    std::function<void(MultiFab& mf, int scomp, int ncomp, Real mean, Real stddev)> fill_normal;
    // one ParallelForRNG launch: z at (i, j, k) of launch `launch`
    std::function<Real(long launch, int i, int j, int k)> point_normal;
    // when set, every draw of a ParallelForRNG body instead: the n-th draw at (i, j, k)
    // of launch `launch`, a uniform (normal = 0) or a standard normal (normal = 1)
    std::function<Real(long launch, int i, int j, int k, long n, int normal)> stream;
    long launches = 0;
};
inline NoiseSource& noise_source() {
    static NoiseSource s;
    return s;
}

struct RandomEngine {
    long launch;
    int i, j, k;
    mutable long n = 0;   // draws made so far at this point
};
inline Real RandomNormal(Real mean, Real stddev, const RandomEngine& e) {
    if (noise_source().stream) return mean + stddev * noise_source().stream(e.launch, e.i, e.j, e.k, e.n++, 1);
    if (!noise_source().point_normal) Abort("RandomNormal: no injected noise source");
    return mean + stddev * noise_source().point_normal(e.launch, e.i, e.j, e.k);
}
inline Real RandomNormal(Real, Real) { Abort("RandomNormal: host-RNG draws are not injected"); }
inline Real Random() { Abort("amrex::Random: uniform draws are not injected"); }
inline Real Random(const RandomEngine& e) {
    if (noise_source().stream) return noise_source().stream(e.launch, e.i, e.j, e.k, e.n++, 0);
    Abort("amrex::Random: uniform draws are not injected");
}
inline unsigned int RandomPoisson(Real, const RandomEngine&) { Abort("amrex::RandomPoisson: not injected"); }
inline unsigned int Random_int(unsigned int, const RandomEngine&) { Abort("amrex::Random_int: not injected"); }

class MFIter;

class MultiFab {
public:
    BoxArray ba;
    DistributionMapping dm;
    int ncomp = 0;
    IntVect ngrow;
    FArrayBox fab;

    MultiFab() = default;
    MultiFab(const BoxArray& b, const DistributionMapping& d, int nc, int ng) { define(b, d, nc, ng); }
    MultiFab(const BoxArray& b, const DistributionMapping& d, int nc, const IntVect& ng) { define(b, d, nc, ng); }
    MultiFab(const BoxArray& b, const DistributionMapping& d, int nc, int ng, const struct MFInfo&) {
        define(b, d, nc, ng);
    }
    MultiFab(const MultiFab&) = delete;
    MultiFab& operator=(const MultiFab&) = delete;
    MultiFab(MultiFab&&) = default;
    MultiFab& operator=(MultiFab&&) = default;

    void define(const BoxArray& b, const DistributionMapping& d, int nc, int ng) { define(b, d, nc, IntVect(ng)); }
    void define(const BoxArray& b, const DistributionMapping& d, int nc, const IntVect& ng) {
        ba = b;
        dm = d;
        ncomp = nc;
        ngrow = ng;
        Box gb = b[0];
        gb.grow(ng);
        fab.resize(gb, nc);
        // AMReX leaves new data uninitialised; NaN makes any read of it visible
        fab.setVal(std::numeric_limits<Real>::quiet_NaN());
    }
    // a MultiFab over caller-owned storage (the harness's Array4-layout buffers)
    void wrap(Real* p, const Box& valid, int nc, int ng) {
        ba = BoxArray(valid);
        ncomp = nc;
        ngrow = IntVect(ng);
        Box gb = valid;
        gb.grow(ng);
        fab.wrap(p, gb, nc);
    }
    bool ok() const { return ba.size() == 1; }
    const BoxArray& boxArray() const { return ba; }
    const DistributionMapping& DistributionMap() const { return dm; }
    int nComp() const { return ncomp; }
    int nGrow(int d = 0) const { return ngrow[d]; }
    IntVect nGrowVect() const { return ngrow; }
    IndexType ixType() const { return ba.ixType(); }
    bool is_nodal(int d) const { return ixType().nodeCentered(d); }
    bool is_cell_centered() const { return ixType().cellCentered(); }
    int size() const { return 1; }
    int local_size() const { return 1; }
    Box box(int) const { return ba[0]; }
    Box fabbox(int) const { return fab.box(); }

    FArrayBox& operator[](const MFIter&) { return fab; }
    const FArrayBox& operator[](const MFIter&) const { return fab; }
    FArrayBox& operator[](int) { return fab; }
    const FArrayBox& operator[](int) const { return fab; }
    Array4<Real> array(const MFIter&) { return fab.array(); }
    Array4<Real const> array(const MFIter&) const { return fab.array(); }
    Array4<Real const> const_array(const MFIter&) const { return fab.array(); }
    Array4<Real> array(int) { return fab.array(); }
    Array4<Real const> const_array(int) const { return fab.array(); }

    template <class F>
    void for_points(int ng, F&& f) const {  // valid box grown by ng (clipped to storage)
        Box b = ba[0];
        b.grow(std::min(ng, ngrow[0]));
        for (int k = b.lo[2]; k <= b.hi[2]; ++k)
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
    }
    void setVal(Real v) { fab.setVal(v); }
    void setVal(Real v, int nghost) { setVal(v, 0, ncomp, nghost); }
    void setVal(Real v, const IntVect& nghost) { setVal(v, 0, ncomp, nghost[0]); }
    void setVal(Real v, int comp, int nc, int nghost) {
        auto a = fab.array();
        for (int n = comp; n < comp + nc; ++n) for_points(nghost, [&](int i, int j, int k) { a(i, j, k, n) = v; });
    }
    void setVal(Real v, int comp, int nc, const IntVect& nghost) { setVal(v, comp, nc, nghost[0]); }
    void mult(Real v, int comp, int nc, int nghost = 0) {
        auto a = fab.array();
        for (int n = comp; n < comp + nc; ++n) for_points(nghost, [&](int i, int j, int k) { a(i, j, k, n) *= v; });
    }
    void mult(Real v, int nghost = 0) { mult(v, 0, ncomp, nghost); }
    void plus(Real v, int comp, int nc, int nghost = 0) {
        auto a = fab.array();
        for (int n = comp; n < comp + nc; ++n) for_points(nghost, [&](int i, int j, int k) { a(i, j, k, n) += v; });
    }
    static void LinComb(MultiFab& dst, Real a, const MultiFab& x, int xcomp, Real b, const MultiFab& y, int ycomp,
                        int dstcomp, int numcomp, int nghost) {
        auto d = dst.fab.array();
        auto xa = x.fab.array();
        auto ya = y.fab.array();
        for (int n = 0; n < numcomp; ++n)
            dst.for_points(nghost, [&](int i, int j, int k) {
                d(i, j, k, dstcomp + n) = a * xa(i, j, k, xcomp + n) + b * ya(i, j, k, ycomp + n);
            });
    }
    static void Copy(MultiFab& dst, const MultiFab& src, int srccomp, int dstcomp, int numcomp, int nghost) {
        auto d = dst.fab.array();
        auto s = src.fab.array();
        for (int n = 0; n < numcomp; ++n)
            dst.for_points(nghost, [&](int i, int j, int k) { d(i, j, k, dstcomp + n) = s(i, j, k, srccomp + n); });
    }
    static void Copy(MultiFab& dst, const MultiFab& src, int srccomp, int dstcomp, int numcomp, const IntVect& ng) {
        Copy(dst, src, srccomp, dstcomp, numcomp, ng[0]);
    }
    static void Add(MultiFab& dst, const MultiFab& src, int srccomp, int dstcomp, int numcomp, int nghost) {
        auto d = dst.fab.array();
        auto s = src.fab.array();
        for (int n = 0; n < numcomp; ++n)
            dst.for_points(nghost, [&](int i, int j, int k) { d(i, j, k, dstcomp + n) += s(i, j, k, srccomp + n); });
    }
    static void Subtract(MultiFab& dst, const MultiFab& src, int srccomp, int dstcomp, int numcomp, int nghost) {
        auto d = dst.fab.array();
        auto s = src.fab.array();
        for (int n = 0; n < numcomp; ++n)
            dst.for_points(nghost, [&](int i, int j, int k) { d(i, j, k, dstcomp + n) -= s(i, j, k, srccomp + n); });
    }
    static void Saxpy(MultiFab& dst, Real a, const MultiFab& src, int srccomp, int dstcomp, int numcomp, int nghost) {
        auto d = dst.fab.array();
        auto s = src.fab.array();
        for (int n = 0; n < numcomp; ++n)
            dst.for_points(nghost, [&](int i, int j, int k) { d(i, j, k, dstcomp + n) += a * s(i, j, k, srccomp + n); });
    }
    Real sum(int comp = 0) const {  // valid region, the reference's loop order
        Real s = 0;
        auto a = fab.array();
        for_points(0, [&](int i, int j, int k) { s += a(i, j, k, comp); });
        return s;
    }
    Real max(int comp, int nghost = 0) const {
        Real m = -std::numeric_limits<Real>::max();
        auto a = fab.array();
        for_points(nghost, [&](int i, int j, int k) { m = std::max(m, a(i, j, k, comp)); });
        return m;
    }
    Real min(int comp, int nghost = 0) const {
        Real m = std::numeric_limits<Real>::max();
        auto a = fab.array();
        for_points(nghost, [&](int i, int j, int k) { m = std::min(m, a(i, j, k, comp)); });
        return m;
    }

    // periodic images of the ghost points, every component
    void FillBoundary(const Periodicity& per, bool = false) { FillBoundary(0, ncomp, per); }
    void FillBoundary(int scomp, int nc, const Periodicity& per, bool = false) {
        const Box v = ba[0];
        const Box g = fab.box();
        auto a = fab.array();
        for (int n = scomp; n < scomp + nc; ++n)
            for (int k = g.lo[2]; k <= g.hi[2]; ++k)
                for (int j = g.lo[1]; j <= g.hi[1]; ++j)
                    for (int i = g.lo[0]; i <= g.hi[0]; ++i) {
                        int p[3] = {i, j, k};
                        bool ghost = false, ok = true;
                        for (int d = 0; d < 3; ++d) {
                            if (p[d] >= v.lo[d] && p[d] <= v.hi[d]) continue;
                            ghost = true;
                            const int L = per.period[d];
                            if (L == 0) { ok = false; break; }
                            while (p[d] < v.lo[d]) p[d] += L;
                            while (p[d] > v.hi[d]) p[d] -= L;
                        }
                        if (ghost && ok) a(i, j, k, n) = a(p[0], p[1], p[2], n);
                    }
    }
    void FillBoundary(int scomp, int nc, const IntVect&, const Periodicity& per, bool = false) {
        FillBoundary(scomp, nc, per);
    }
    // nodal periodic duplicates: the high boundary point takes the low one's value
    // Multi-box machinery that only ComputeAverages.cpp's slice, pencil and
    // column functions name (not part of the host build: a call reports itself).
    std::vector<Array4<Real const>> const_arrays() const { Abort("MultiFab::const_arrays: multi-box API"); }
    void setFab(int, FArrayBox&&) { Abort("MultiFab::setFab: multi-box API"); }
    void ParallelAdd(const MultiFab&) { Abort("MultiFab::ParallelAdd: multi-box API"); }
    void ParallelCopy(const MultiFab&, int = 0, int = 0, int = 0) { Abort("MultiFab::ParallelCopy: multi-box API"); }
    void OverrideSync(const Periodicity& per) {
        const Box v = ba[0];
        auto a = fab.array();
        const IntVect t = v.typ.t;
        for (int n = 0; n < ncomp; ++n)
            for (int k = v.lo[2]; k <= v.hi[2]; ++k)
                for (int j = v.lo[1]; j <= v.hi[1]; ++j)
                    for (int i = v.lo[0]; i <= v.hi[0]; ++i) {
                        int p[3] = {i, j, k};
                        bool dup = false;
                        for (int d = 0; d < 3; ++d)
                            if (t[d] == 1 && per.period[d] != 0 && p[d] == v.hi[d]) { p[d] = v.lo[d]; dup = true; }
                        if (dup) a(i, j, k, n) = a(p[0], p[1], p[2], n);
                    }
    }
};

inline int TilingIfNotGPU() { return 0; }

class MFIter {
public:
    const MultiFab* mf;
    bool valid = true;
    MFIter(const MultiFab& m, bool = false) : mf(&m) {}
    MFIter(const MultiFab& m, int) : mf(&m) {}
    MFIter(const MultiFab& m, const IntVect&) : mf(&m) {}
    MFIter(const BoxArray&, const DistributionMapping&, bool = false) : mf(nullptr) {
        Abort("MFIter over a BoxArray is not supported by the host stand-in");
    }
    bool isValid() const { return valid; }
    void operator++() { valid = false; }
    int index() const { return 0; }
    int LocalIndex() const { return 0; }
    Box validbox() const { return mf->ba[0]; }
    Box tilebox() const { return validbox(); }
    Box tilebox(const IntVect& nodal) const { return convert(validbox(), nodal); }
    Box tilebox(const IntVect& nodal, const IntVect& ng) const { return grow(convert(validbox(), nodal), ng); }
    Box nodaltilebox(int d) const { return surroundingNodes(validbox(), d); }
    Box growntilebox(int ng) const { return grow(validbox(), ng); }
    Box growntilebox(const IntVect& ng) const { return grow(validbox(), ng); }
    Box grownnodaltilebox(int d, int ng) const { return grow(surroundingNodes(validbox(), d), ng); }
    Box fabbox() const { return mf->fab.box(); }
};

// ---- loops --------------------------------------------------------------------------
template <class F>
inline void LoopBox(const Box& b, F&& f) {
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}
template <class F>
inline void ParallelFor(const Box& b, F&& f) { LoopBox(b, f); }
template <class F>
inline void ParallelFor(const Box& b, int nc, F&& f) {
    for (int n = 0; n < nc; ++n) LoopBox(b, [&](int i, int j, int k) { f(i, j, k, n); });
}
template <class F1, class F2>
inline void ParallelFor(const Box& b1, const Box& b2, F1&& f1, F2&& f2) {
    LoopBox(b1, f1);
    LoopBox(b2, f2);
}
template <class F1, class F2, class F3>
inline void ParallelFor(const Box& b1, const Box& b2, const Box& b3, F1&& f1, F2&& f2, F3&& f3) {
    LoopBox(b1, f1);
    LoopBox(b2, f2);
    LoopBox(b3, f3);
}
template <class F1, class F2, class F3>
inline void ParallelFor(const Box& b1, int n1, F1&& f1, const Box& b2, int n2, F2&& f2, const Box& b3, int n3,
                        F3&& f3) {
    ParallelFor(b1, n1, f1);
    ParallelFor(b2, n2, f2);
    ParallelFor(b3, n3, f3);
}
template <class F>
inline void ParallelFor(Long n, F&& f) { for (Long q = 0; q < n; ++q) f(q); }
template <class F>
inline void ParallelForRNG(const Box& b, F&& f) {
    const long launch = noise_source().launches++;
    LoopBox(b, [&](int i, int j, int k) { f(i, j, k, RandomEngine{launch, i, j, k, 0}); });
}

inline void FillRandomNormal(MultiFab& mf, int scomp, int ncomp, Real mean, Real stddev) {
    if (!noise_source().fill_normal) Abort("FillRandomNormal: no injected noise source");
    noise_source().fill_normal(mf, scomp, ncomp, mean, stddev);
}
inline void FillRandom(MultiFab&, int, int) { Abort("FillRandom: uniform draws are not injected"); }

// ---- single process -----------------------------------------------------------------
namespace ParallelDescriptor {
inline int MyProc() { return 0; }
inline int NProcs() { return 1; }
inline int IOProcessorNumber() { return 0; }
inline bool IOProcessor() { return true; }
inline double second() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
template <class T> inline void ReduceRealSum(T&, int = 0) {}
inline void ReduceRealSum(Real*, int, int = 0) {}
template <class T> inline void ReduceRealMax(T&, int = 0) {}
template <class T> inline void ReduceRealMin(T&, int = 0) {}
template <class T> inline void ReduceIntSum(T&, int = 0) {}
template <class T> inline void ReduceIntMax(T&, int = 0) {}
template <class T> inline void ReduceLongSum(T&, int = 0) {}
template <class T> inline void Bcast(T*, size_t, int = 0) {}
inline void Barrier() {}
}  // namespace ParallelDescriptor

// ---- ParmParse over an in-memory table ------------------------------------------------
class ParmParse {
public:
    static std::map<std::string, std::vector<std::string>>& table() {
        static std::map<std::string, std::vector<std::string>> t;
        return t;
    }
    // "key = v1 v2 ..." lines; '#' starts a comment
    static void load(const std::string& text) {
        table().clear();
        std::istringstream is(text);
        std::string line;
        while (std::getline(is, line)) {
            const size_t h = line.find('#');
            if (h != std::string::npos) line.resize(h);
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            std::istringstream ks(line.substr(0, eq)), vs(line.substr(eq + 1));
            std::string key, v;
            ks >> key;
            std::vector<std::string> vals;
            while (vs >> v) vals.push_back(v);
            if (!key.empty()) table()[key] = vals;
        }
    }
    std::string prefix;
    ParmParse() = default;
    explicit ParmParse(const std::string& p) : prefix(p) {}
    std::string full(const std::string& k) const { return prefix.empty() ? k : prefix + "." + k; }
    const std::vector<std::string>* find(const std::string& k) const {
        auto it = table().find(full(k));
        return it == table().end() ? nullptr : &it->second;
    }
    bool contains(const std::string& k) const { return find(k) != nullptr; }
    int countval(const std::string& k) const { auto v = find(k); return v ? (int)v->size() : 0; }

    static void conv(const std::string& s, int& v) { v = std::stoi(s); }
    static void conv(const std::string& s, long& v) { v = std::stol(s); }
    static void conv(const std::string& s, long long& v) { v = std::stoll(s); }
    static void conv(const std::string& s, double& v) { v = std::stod(s); }
    static void conv(const std::string& s, float& v) { v = std::stof(s); }
    static void conv(const std::string& s, std::string& v) { v = s; }
    static void conv(const std::string& s, bool& v) {
        v = (s == "1" || s == "true" || s == "True" || s == "TRUE" || s == "t" || s == "T");
    }
    template <class T>
    bool query(const std::string& k, T& v, int ival = 0) const {
        auto vals = find(k);
        if (!vals || (int)vals->size() <= ival) return false;
        conv((*vals)[ival], v);
        return true;
    }
    template <class T>
    void get(const std::string& k, T& v, int ival = 0) const {
        if (!query(k, v, ival)) Abort("ParmParse::get: missing " + full(k));
    }
    template <class T>
    bool queryarr(const std::string& k, std::vector<T>& v, int start = 0, int n = -1) const {
        auto vals = find(k);
        if (!vals) return false;
        if (n < 0) n = (int)vals->size() - start;
        if ((int)vals->size() < start + n) Abort("ParmParse::queryarr: too few values for " + full(k));
        v.resize(n);
        for (int q = 0; q < n; ++q) { T x; conv((*vals)[start + q], x); v[q] = x; }
        return true;
    }
    template <class T>
    void getarr(const std::string& k, std::vector<T>& v, int start = 0, int n = -1) const {
        if (!queryarr(k, v, start, n)) Abort("ParmParse::getarr: missing " + full(k));
    }
    template <class T, size_t N>
    bool queryarr(const std::string& k, std::array<T, N>& v, int start = 0, int n = (int)N) const {
        std::vector<T> t;
        if (!queryarr(k, t, start, n)) return false;
        for (int q = 0; q < n; ++q) v[q] = t[q];
        return true;
    }
    template <class T>
    void add(const std::string& k, const T& v) {
        std::ostringstream os;
        os << v;
        table()[full(k)] = {os.str()};
    }
};

// ---- names of ComputeAverages.cpp's multi-box functions (not part of the host build) ----
struct MFInfo {
    MFInfo& SetAlloc(bool) { return *this; }
};
struct ReduceOpSum {};
template <class Op, class T, class F>
FArrayBox ReduceToPlane(int, const Box&, const MultiFab&, F&&) {
    Abort("ReduceToPlane: multi-box API");
}

// ---- file names and plotfiles -------------------------------------------------------------
inline std::string Concatenate(const std::string& root, int num, int mindigits = 5) {
    std::ostringstream os;
    os << root << std::setfill('0') << std::setw(mindigits) << num;
    return os.str();
}
struct CoordSys {
    enum CoordType { undef = -1, cartesian = 0, RZ = 1, SPHERICAL = 2 };
};
// WriteSingleLevelPlotfile does not write files here: it keeps the last plotfile
// MultiFab's valid region (Array4 order, component slowest), its names, time and
// step, which the harness reads back (the on-disk format is AMReX's, not the
// reference's).
struct PlotfileCapture {
    std::string name;
    std::vector<Real> data;
    std::vector<std::string> names;
    Real time = 0;
    int step = 0;
};
inline PlotfileCapture& plotfile_capture() {
    static PlotfileCapture c;
    return c;
}
inline void WriteSingleLevelPlotfile(const std::string& name, const MultiFab& mf, const Vector<std::string>& names,
                                     const Geometry&, Real time, int step) {
    PlotfileCapture& c = plotfile_capture();
    c.name = name;
    c.names.assign(names.begin(), names.end());
    c.time = time;
    c.step = step;
    c.data.clear();
    const Box v = mf.boxArray()[0];
    const auto a = mf.const_array(0);
    for (int n = 0; n < mf.nComp(); ++n)
        for (int k = v.lo[2]; k <= v.hi[2]; ++k)
            for (int j = v.lo[1]; j <= v.hi[1]; ++j)
                for (int i = v.lo[0]; i <= v.hi[0]; ++i) c.data.push_back(a(i, j, k, n));
}

// ---- sumToLine (one box, one process: the reduction over ranks is the identity) -------
inline Gpu::HostVector<Real> sumToLine(const MultiFab& mf, int icomp, int ncomp, const Box& domain, int direction,
                                       bool /*local*/ = false) {
    Gpu::HostVector<Real> hv((size_t)domain.length(direction) * ncomp, 0.0);
    const Box b = mf.boxArray()[0];
    const auto a = mf.const_array(0);
    for (int n = 0; n < ncomp; ++n)
        for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
            for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
                for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
                    const int m = (direction == 0 ? i : direction == 1 ? j : k) - domain.smallEnd(direction);
                    hv[(size_t)m * ncomp + n] += a(i, j, k, icomp + n);
                }
    return hv;
}

// ---- VisMF and plotfiles: not part of the step ------------------------------------------
struct VisMF {
    template <class... A> static void Write(const A&...) { Abort("VisMF::Write is not supported by the host stand-in"); }
    template <class... A> static void Read(A&...) { Abort("VisMF::Read is not supported by the host stand-in"); }
};

}  // namespace amrex

// BC type constants used by the boundary routines' headers
namespace amrex {
namespace BCType {
enum mathematicalBndryTypes : int {
    bogus = -666, reflect_odd = -1, int_dir = 0, reflect_even = 1, foextrap = 2, ext_dir = 3, hoextrap = 4,
    Interior = 0, Inflow = 1, Outflow = 2, Symmetry = 3, SlipWall = 4, NoSlipWall = 5
};
}
class BCRec {
public:
    int bc[6] = {0, 0, 0, 0, 0, 0};
    const int* lo() const { return bc; }
    const int* hi() const { return bc + 3; }
    int lo(int d) const { return bc[d]; }
    int hi(int d) const { return bc[3 + d]; }
    void setLo(int d, int v) { bc[d] = v; }
    void setHi(int d, int v) { bc[3 + d] = v; }
};
}  // namespace amrex
