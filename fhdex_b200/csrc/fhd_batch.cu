// fhd_batch.cu — many independent runs (ensemble members or served requests) of one
// species count and precision advanced together: every kernel of the RK3 step is
// launched once for all members (block -> member lookup), and one step is
// replayed from a captured CUDA graph.  Members may have different box sizes,
// gas states, time steps, seeds and step counters; each member's result is the
// same as that run alone through fhd_rk3_step_stag (same kernels, same operation
// order, same per-member Philox key and counters).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "fhd_host.h"

using namespace fhd;

namespace {

const int NGC = 2;
const int CELLN[3] = {0, 0, 0};
const int ALLN[3] = {1, 1, 1};
const int FACEN[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

int64_t pts(const fhd_fab& f) {
    int64_t n = 1;
    for (int d = 0; d < 3; ++d) n *= (int64_t)(f.hi[d] - f.lo[d] + 1);
    return n;
}

fhd_fab mk(const int n[3], const int nodal[3], int ng, int nc, int dtype) {
    fhd_fab f;
    f.data = nullptr;
    for (int d = 0; d < 3; ++d) {
        f.lo[d] = -ng;
        f.hi[d] = n[d] - 1 + nodal[d] + ng;
        f.nodal[d] = nodal[d];
    }
    f.ncomp = nc;
    f.dtype = dtype;
    return f;
}

bool geom_ok(const fhd_fab& f, const int n[3], const int nodal[3], int ng, int min_nc) {
    if (!f.data || f.dtype != FHD_F64 || f.ncomp < min_nc) return false;
    for (int d = 0; d < 3; ++d)
        if (f.lo[d] != -ng || f.hi[d] != n[d] - 1 + nodal[d] + ng || f.nodal[d] != nodal[d]) return false;
    return pts(f) * f.ncomp < ((int64_t)1 << 31);
}


struct Member {
    int id = -1;
    fhd_params prm{};
    double dt = 0;
    uint64_t step = 0;          // next step number (host copy)
    fhd_fab cu{}, mom[3]{}, prim{}, vel[3]{};
    void* scratch = nullptr;
    size_t bytes = 0;
    fhd_fab cup{}, cup2{}, cupm[3]{}, cup2m[3]{}, eta{}, zeta{}, kappa{}, chi{}, D{}, ct{}, et{}, sff[3]{}, smc{}, sme{};
    int64_t cells = 0;
};

struct Launch {
    int kind;          // 0..6 kernel kind, 7 ghost fill, 8 step increment
    size_t args_off;   // offset of the packed argument array in the device buffer
    size_t bpref_off;  // offset of the block-prefix array
    int nitems;        // members (or fabs)
    int nblocks;
    size_t stride;     // bytes of one member's (fab's) argument block
    std::vector<int64_t> items;  // work items per member (fab)
};

// items per chunk of the persistent step (k_batch_persist)
const int kPersistChunk = 2048;

const double kW[3] = {(2.0 * std::sqrt(2.0) + 1.0 * std::sqrt(3.0)) / 5.0,
                      (-4.0 * std::sqrt(2.0) + 3.0 * std::sqrt(3.0)) / 5.0,
                      (1.0 * std::sqrt(2.0) - 2.0 * std::sqrt(3.0)) / 10.0};

}  // namespace

struct fhd_batch {
    int device = 0, ns = 2;
    bool mixed = false;
    int mode = -1;  // NM_PHILOX or NM_OFF, fixed by the first member
    cudaStream_t own = nullptr, stream = nullptr;
    std::vector<Member> mem;
    int next_id = 0;
    bool dirty = true;
    // device plan
    void* dbuf = nullptr;
    size_t dbuf_bytes = 0;
    uint64_t* dsteps = nullptr;  // inside dbuf
    int* dstatus = nullptr;      // inside dbuf, one word per member
    std::vector<Launch> plan;
    int tile = -1;               // face-kernel register cap (batch_face_tiles(); -1 default)
    // the persistent step: one launch per RK3 step over a work-unit table in dbuf
    bool persistent = false;
    PersistArgs pargs{};
    size_t counters_bytes = 0;   // next, abort, done[] (zeroed before each launch)
    double wait_limit_s = 1.0;
    int hold_phase = -1;
    int persist_tile = -1;       // register cap of the persistent kernel (batch face tiles; -1 default)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
};

namespace {

int cuda_ok(cudaError_t e) {
    if (e == cudaSuccess) return FHD_OK;
    cudaGetLastError();
    return FHD_ERR_CUDA;
}

void drop_graph(fhd_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

// stage scratch of one member, carved from one stream-ordered allocation
int alloc_member(fhd_batch* b, Member& m) {
    const int* n = m.prm.n_cells;
    const int ns = b->ns;
    const int rdt = b->mixed ? FHD_F32 : FHD_F64;
    const size_t re = b->mixed ? 4 : 8;
    m.cup = mk(n, CELLN, NGC, 5 + ns, FHD_F64);
    m.cup2 = m.cup;
    for (int d = 0; d < 3; ++d) m.cupm[d] = m.cup2m[d] = mk(n, FACEN[d], NGC, 1, FHD_F64);
    m.eta = mk(n, CELLN, NGC, 1, rdt);
    m.zeta = m.eta;
    m.kappa = m.eta;
    m.chi = mk(n, CELLN, NGC, ns, rdt);
    m.D = mk(n, CELLN, NGC, ns * ns, rdt);
    m.ct = mk(n, CELLN, 1, 6, rdt);
    m.et = mk(n, ALLN, 0, 6, rdt);
    for (int d = 0; d < 3; ++d) m.sff[d] = mk(n, ALLN, 0, 2 + ns, FHD_F64);
    m.smc = mk(n, CELLN, 1, 3, FHD_F64);
    m.sme = mk(n, ALLN, 0, 6, FHD_F64);
    struct P { fhd_fab* f; size_t e; } parts[] = {
        {&m.cup, 8}, {&m.cup2, 8}, {&m.cupm[0], 8}, {&m.cupm[1], 8}, {&m.cupm[2], 8}, {&m.cup2m[0], 8},
        {&m.cup2m[1], 8}, {&m.cup2m[2], 8}, {&m.eta, re}, {&m.zeta, re}, {&m.kappa, re}, {&m.chi, re}, {&m.D, re},
        {&m.ct, re}, {&m.et, re}, {&m.sff[0], 8}, {&m.sff[1], 8}, {&m.sff[2], 8}, {&m.smc, 8}, {&m.sme, 8}};
    size_t total = 0;
    for (auto& q : parts) total += ((size_t)pts(*q.f) * q.f->ncomp * q.e + 255) & ~(size_t)255;
    if (cudaMallocAsync(&m.scratch, total, b->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
    m.bytes = total;
    char* p = static_cast<char*>(m.scratch);
    for (auto& q : parts) {
        q.f->data = p;
        p += ((size_t)pts(*q.f) * q.f->ncomp * q.e + 255) & ~(size_t)255;
    }
    return FHD_OK;
}

// one member's StageCall for stage s (0..2)
StageCall member_call(const fhd_batch* b, const Member& m, int s, const uint64_t* dstep, int* dstatus) {
    StageCall sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.P = dev_params(m.prm, m.dt, m.step);
    sc.P.step_ptr = dstep;
    sc.mode = b->mode;
    sc.w = kW[s];
    sc.stage = s + 1;
    const fhd_fab* ins[3] = {&m.cu, &m.cup, &m.cup2};
    const fhd_fab* insm[3] = {m.mom, m.cupm, m.cup2m};
    const fhd_fab* outs[3] = {&m.cup, &m.cup2, &m.cu};
    const fhd_fab* outsm[3] = {m.cupm, m.cup2m, m.mom};
    sc.cons_s = *ins[s];
    sc.cons_o = *outs[s];
    sc.cons0 = m.cu;
    for (int d = 0; d < 3; ++d) {
        sc.mom_s[d] = insm[s][d];
        sc.mom_o[d] = outsm[s][d];
        sc.mom0[d] = m.mom[d];
        sc.vel[d] = m.vel[d];
        sc.sff[d] = m.sff[d];
    }
    sc.pr = m.prim;
    sc.pT = 4;
    sc.eta = m.eta; sc.zeta = m.zeta; sc.kappa = m.kappa; sc.chi = m.chi; sc.D = m.D;
    sc.ct = m.ct;
    sc.et = m.et;
    sc.smc = m.smc;
    sc.sme = m.sme;
    sc.status = dstatus;
    sc.tile = 0;
    return sc;
}

int64_t kind_items(int kind, const int n[3]) {
    switch (kind) {
        case 0: return (int64_t)(n[0] + 3) * (n[1] + 3) * (n[2] + 3);
        case 1: return (int64_t)(n[0] + 2) * (n[1] + 2) * (n[2] + 2);
        case 2: return (int64_t)(n[0] + 1) * n[1] * n[2];
        case 3: return (int64_t)n[0] * (n[1] + 1) * n[2];
        case 4: return (int64_t)n[0] * n[1] * (n[2] + 1);
        case 5: return (int64_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1);
        case 6: return (int64_t)n[0] * n[1] * n[2];
        default: return 0;
    }
}

// Builds the per-member argument arrays, block prefixes and launch plan of one RK3
// step, and uploads them (synchronously with respect to the batch stream).
int rebuild(fhd_batch* b) {
    drop_graph(b);
    b->plan.clear();
    const int M = (int)b->mem.size();
    if (M == 0) { b->dirty = false; return FHD_OK; }
    std::vector<char> host;
    auto align = [&](size_t a) { size_t o = (host.size() + a - 1) & ~(a - 1); host.resize(o); return o; };
    // steps and statuses first
    const size_t steps_off = align(256);
    host.resize(steps_off + sizeof(uint64_t) * M);
    for (int q = 0; q < M; ++q) memcpy(host.data() + steps_off + sizeof(uint64_t) * q, &b->mem[q].step, sizeof(uint64_t));
    const size_t status_off = align(256);
    host.resize(status_off + sizeof(int) * M, 0);
    // the argument structs embed device pointers to the step and status words, so the
    // buffer is sized and allocated before anything is packed
    const int ghost_sz = ghost_desc_size();
    size_t need = host.size();
    auto add = [&](size_t bytes) { need = ((need + 255) & ~(size_t)255) + bytes; };
    for (int s = 0; s < 3; ++s) {
        add(batch_args_size(b->ns, b->mixed, 0, b->mode) * M);
        add(batch_args_size(b->ns, b->mixed, 1, b->mode) * M);
        for (int kind = 0; kind < 6; ++kind) add(sizeof(int) * (M + 1));
        add((size_t)ghost_sz * 5 * M);
        add(sizeof(int) * (5 * M + 1));
    }
    add(batch_args_size(b->ns, false, 6, b->mode) * M);
    add(sizeof(int) * (M + 1));
    add((size_t)ghost_sz * 5 * M);
    add(sizeof(int) * (5 * M + 1));
    // persistent step: 24 phases; 11 units per member and stage, 7 for the end
    const int kPhases = 24;
    add(sizeof(PUnit) * (size_t)40 * M);
    add(sizeof(unsigned int) * (size_t)kPhases * M);
    add(sizeof(unsigned int) * ((size_t)kPhases * M + 2));
    need += 4096;
    if (!b->dbuf || b->dbuf_bytes < need) {
        if (b->dbuf) cudaFreeAsync(b->dbuf, b->stream);
        b->dbuf = nullptr;
        if (cudaMallocAsync(&b->dbuf, need, b->stream) != cudaSuccess) { cudaGetLastError(); return FHD_ERR_OOM; }
        b->dbuf_bytes = need;
    }
    char* dbase = static_cast<char*>(b->dbuf);
    b->dsteps = reinterpret_cast<uint64_t*>(dbase + steps_off);
    b->dstatus = reinterpret_cast<int*>(dbase + status_off);
    auto push_bpref = [&](const std::vector<int64_t>& items, int bs, int& nblocks) {
        std::vector<int> pref(items.size() + 1, 0);
        for (size_t q = 0; q < items.size(); ++q) pref[q + 1] = pref[q] + (int)((items[q] + bs - 1) / bs);
        nblocks = pref.back();
        const size_t off = align(256);
        host.resize(off + sizeof(int) * pref.size());
        memcpy(host.data() + off, pref.data(), sizeof(int) * pref.size());
        return off;
    };
    auto push_args = [&](int kind, bool mixed, int s) {
        const size_t sz = batch_args_size(b->ns, mixed, kind, b->mode);
        const size_t off = align(256);
        host.resize(off + sz * M);
        for (int q = 0; q < M; ++q) {
            const Member& m = b->mem[q];
            StageCall sc = member_call(b, m, s, b->dsteps + q, b->dstatus + q);
            if (kind == 6) { sc.pr = m.prim; sc.cons_o = m.cu; for (int d = 0; d < 3; ++d) sc.mom_o[d] = m.mom[d]; }
            batch_pack(b->ns, mixed, kind, b->mode, sc, host.data() + off + sz * q);
        }
        return off;
    };
    auto push_ghosts = [&](int s, int& nfab, int& nblocks, std::vector<int64_t>& items) {
        const size_t off = align(256);
        host.resize(off + (size_t)ghost_sz * 5 * M);
        items.clear();
        int f = 0;
        for (int q = 0; q < M; ++q) {
            const Member& m = b->mem[q];
            const int* n = m.prm.n_cells;
            const fhd_fab* o = (s == 0) ? &m.cup : (s == 1) ? &m.cup2 : &m.cu;
            const fhd_fab* om = (s == 0) ? m.cupm : (s == 1) ? m.cup2m : m.mom;
            if (s < 3) {
                items.push_back(ghost_pack(*o, 0, 1, n, host.data() + off + (size_t)ghost_sz * f++));
                items.push_back(ghost_pack(*o, 4, 1 + b->ns, n, host.data() + off + (size_t)ghost_sz * f++));
                for (int d = 0; d < 3; ++d)
                    items.push_back(ghost_pack(om[d], 0, 1, n, host.data() + off + (size_t)ghost_sz * f++));
            }
        }
        nfab = f;
        const size_t bpo = push_bpref(items, 256, nblocks);
        return std::make_pair(off, bpo);
    };
    auto push_final_ghosts = [&](int& nfab, int& nblocks, std::vector<int64_t>& items) {
        const size_t off = align(256);
        host.resize(off + (size_t)ghost_sz * 5 * M);
        items.clear();
        int f = 0;
        for (int q = 0; q < M; ++q) {
            const Member& m = b->mem[q];
            const int* n = m.prm.n_cells;
            items.push_back(ghost_pack(m.cu, 1, 3, n, host.data() + off + (size_t)ghost_sz * f++));
            items.push_back(ghost_pack(m.prim, 0, 6 + 2 * b->ns, n, host.data() + off + (size_t)ghost_sz * f++));
            for (int d = 0; d < 3; ++d)
                items.push_back(ghost_pack(m.vel[d], 0, 1, n, host.data() + off + (size_t)ghost_sz * f++));
        }
        nfab = f;
        const size_t bpo = push_bpref(items, 256, nblocks);
        return std::make_pair(off, bpo);
    };
    for (int s = 0; s < 3; ++s) {
        const size_t prep = push_args(0, b->mixed, s);
        const size_t stg = push_args(1, b->mixed, s);
        for (int kind = 0; kind <= 5; ++kind) {
            std::vector<int64_t> items;
            for (const Member& m : b->mem) items.push_back(kind_items(kind, m.prm.n_cells));
            int nb = 0;
            const size_t bpo = push_bpref(items, 128, nb);
            b->plan.push_back(Launch{kind, kind == 0 ? prep : stg, bpo, M, nb,
                                     batch_args_size(b->ns, b->mixed, kind == 0 ? 0 : 1, b->mode), items});
        }
        int nfab = 0, nb = 0;
        std::vector<int64_t> gitems;
        auto g = push_ghosts(s, nfab, nb, gitems);
        b->plan.push_back(Launch{7, g.first, g.second, nfab, nb, (size_t)ghost_sz, gitems});
    }
    {
        const size_t conv = push_args(6, false, 2);
        std::vector<int64_t> items;
        for (const Member& m : b->mem) items.push_back(kind_items(6, m.prm.n_cells));
        int nb = 0;
        const size_t bpo = push_bpref(items, 128, nb);
        b->plan.push_back(Launch{6, conv, bpo, M, nb, batch_args_size(b->ns, false, 6, b->mode), items});
        int nfab = 0;
        std::vector<int64_t> gitems;
        auto g = push_final_ghosts(nfab, nb, gitems);
        b->plan.push_back(Launch{7, g.first, g.second, nfab, nb, (size_t)ghost_sz, gitems});
        b->plan.push_back(Launch{8, 0, 0, M, 0, 0, std::vector<int64_t>(M, 1)});
    }
    // the persistent step's work units, phase-major over members, with each
    // member's chunk count per phase and the zeroed counters
    {
        const int nph = (int)b->plan.size();
        std::vector<PUnit> units;
        std::vector<unsigned int> needv((size_t)nph * M, 0);
        int64_t first = 0;
        for (int ph = 0; ph < nph; ++ph) {
            const Launch& L = b->plan[ph];
            const int per = L.kind == 7 ? 5 : 1;  // ghost fabs per member
            for (size_t u = 0; u < L.items.size(); ++u) {
                PUnit pu;
                pu.args = L.kind == 8 ? nullptr : dbase + L.args_off + L.stride * u;
                pu.first = first;
                pu.items = L.items[u];
                pu.member = (int)(u / per);
                pu.phase = ph;
                pu.kind = L.kind;
                pu.pad = 0;
                const int64_t nch = (pu.items + kPersistChunk - 1) / kPersistChunk;
                first += nch;
                needv[(size_t)pu.member * nph + ph] += (unsigned int)nch;
                units.push_back(pu);
            }
        }
        const size_t uoff = align(256);
        host.resize(uoff + sizeof(PUnit) * units.size());
        memcpy(host.data() + uoff, units.data(), sizeof(PUnit) * units.size());
        const size_t noff = align(256);
        host.resize(noff + sizeof(unsigned int) * needv.size());
        memcpy(host.data() + noff, needv.data(), sizeof(unsigned int) * needv.size());
        const size_t coff = align(256);
        b->counters_bytes = sizeof(unsigned int) * (needv.size() + 2);
        host.resize(coff + b->counters_bytes, 0);
        PersistArgs& a = b->pargs;
        a.units = reinterpret_cast<const PUnit*>(dbase + uoff);
        a.nunits = (int)units.size();
        a.nphase = nph;
        a.total = first;
        a.chunk = kPersistChunk;
        a.next = reinterpret_cast<unsigned int*>(dbase + coff);
        a.abort = reinterpret_cast<int*>(dbase + coff + sizeof(unsigned int));
        a.done = reinterpret_cast<unsigned int*>(dbase + coff + 2 * sizeof(unsigned int));
        a.need = reinterpret_cast<const unsigned int*>(dbase + noff);
        a.status = b->dstatus;
        a.steps = b->dsteps;
        a.limit_ns = (unsigned long long)(b->wait_limit_s * 1e9);
        a.hold_phase = b->hold_phase;
    }
    if (host.size() > b->dbuf_bytes) return FHD_ERR_OOM;
    if (cudaMemcpyAsync(b->dbuf, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
        return cuda_ok(cudaGetLastError());
    // the host staging vector dies here: wait for the copy
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return cuda_ok(cudaGetLastError());
    b->dirty = false;
    return FHD_OK;
}

int run_plan(fhd_batch* b) {
    if (b->persistent) {
        // zero the dispenser, the abort flag and the per-phase counters, then one launch
        if (cudaMemsetAsync(b->pargs.next, 0, b->counters_bytes, b->stream) != cudaSuccess)
            return cuda_ok(cudaGetLastError());
        return batch_persist(b->ns, b->mixed, b->mode, b->persist_tile, b->pargs, b->stream);
    }
    char* d = static_cast<char*>(b->dbuf);
    for (const Launch& L : b->plan) {
        int rc = FHD_OK;
        if (L.kind <= 6) {
            const bool mixed = (L.kind == 6) ? false : b->mixed;
            rc = batch_launch(b->ns, mixed, L.kind, b->mode, b->tile, d + L.args_off,
                              reinterpret_cast<const int*>(d + L.bpref_off), L.nitems, L.nblocks, b->stream);
        } else if (L.kind == 7) {
            rc = ghost_launch_b(d + L.args_off, reinterpret_cast<const int*>(d + L.bpref_off), L.nitems, L.nblocks,
                                b->stream);
        } else {
            rc = steps_inc(b->dsteps, L.nitems, b->stream);
        }
        if (rc) return rc;
    }
    return FHD_OK;
}

int find(const fhd_batch* b, int id) {
    for (size_t q = 0; q < b->mem.size(); ++q)
        if (b->mem[q].id == id) return (int)q;
    return -1;
}

// pulls the device step counters back into the members (before a rebuild)
int sync_steps(fhd_batch* b) {
    if (b->mem.empty() || !b->dsteps || b->dirty) return FHD_OK;
    std::vector<uint64_t> s(b->mem.size());
    if (cudaMemcpyAsync(s.data(), b->dsteps, sizeof(uint64_t) * s.size(), cudaMemcpyDeviceToHost, b->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return cuda_ok(cudaGetLastError());
    for (size_t q = 0; q < s.size(); ++q) b->mem[q].step = s[q];
    return FHD_OK;
}

}  // namespace

extern "C" {

int fhd_batch_create(fhd_batch** out, int nspecies, int precision, int device) {
    if (!out) return FHD_ERR_BAD_ARG;
    *out = nullptr;
    if (nspecies < 1 || nspecies > 4) return FHD_ERR_UNSUPPORTED;
    if (precision != FHD_PREC_FP64 && precision != FHD_PREC_MIXED) return FHD_ERR_BAD_ARG;
    fhd_batch* b = new (std::nothrow) fhd_batch;
    if (!b) return FHD_ERR_OOM;
    b->device = device;
    b->ns = nspecies;
    b->mixed = precision == FHD_PREC_MIXED;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return FHD_ERR_CUDA;
    }
    b->stream = b->own;
    *out = b;
    return FHD_OK;
}

int fhd_batch_destroy(fhd_batch* b) {
    if (!b) return FHD_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (Member& m : b->mem)
        if (m.scratch) cudaFreeAsync(m.scratch, b->stream);
    if (b->dbuf) cudaFreeAsync(b->dbuf, b->stream);
    cudaStreamSynchronize(b->stream);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return FHD_OK;
}

int fhd_batch_set_stream(fhd_batch* b, void* stream) {
    if (!b) return FHD_ERR_BAD_ARG;
    b->stream = static_cast<cudaStream_t>(stream);
    drop_graph(b);
    return FHD_OK;
}

int fhd_batch_add(fhd_batch* b, const fhd_params* params, fhd_fab cu, const fhd_fab mom[3], fhd_fab prim,
                  const fhd_fab vel[3], double dt, int64_t first_step, const double* init, int* member) {
    if (!b || !params || !mom || !vel || !member || !(dt > 0)) return FHD_ERR_BAD_ARG;
    fhd_params p = *params;
    if (p.nspecies != b->ns || p.precision != (b->mixed ? FHD_PREC_MIXED : FHD_PREC_FP64)) return FHD_ERR_BAD_ARG;
    if (p.algorithm_type != 2 || p.transport_type != 1 || p.advection_type < -1 || p.advection_type > 2 ||
        (p.stoch_stress_form != 0 && p.stoch_stress_form != 1) || ((p.visc_type == 3 || p.visc_type == -3) && p.zeta_ratio < 0) ||
        p.nreaction != 0 || reference_order(p))
        return FHD_ERR_UNSUPPORTED;
    const int mode = p.stoch_stress_form == 1 ? NM_PHILOX : NM_OFF;
    if (b->mode >= 0 && b->mode != mode && !b->mem.empty()) return FHD_ERR_BAD_ARG;
    const int* n = p.n_cells;
    for (int d = 0; d < 3; ++d)
        if (n[d] < 2 || !(p.prob_hi[d] > p.prob_lo[d])) return FHD_ERR_BAD_ARG;
    if (!geom_ok(cu, n, CELLN, NGC, 5 + b->ns) || !geom_ok(prim, n, CELLN, NGC, 6 + 2 * b->ns)) return FHD_ERR_BAD_ARG;
    for (int d = 0; d < 3; ++d)
        if (!geom_ok(mom[d], n, FACEN[d], NGC, 1) || !geom_ok(vel[d], n, FACEN[d], NGC, 1)) return FHD_ERR_BAD_ARG;
    // GetHcGas (compressible_functions.cpp:91-100)
    for (int i = 0; i < p.nspecies; ++i) {
        if (p.hcv[i] < 0.) p.hcv[i] = 0.5 * p.dof[i] * p.Runiv / p.molmass[i];
        if (p.hcp[i] < 0.) p.hcp[i] = 0.5 * (2. + p.dof[i]) * p.Runiv / p.molmass[i];
    }
    cudaSetDevice(b->device);
    int rc = sync_steps(b);
    if (rc) return rc;
    Member m;
    m.id = b->next_id++;
    m.prm = p;
    m.dt = dt;
    m.step = (uint64_t)first_step;
    m.cu = cu;
    m.prim = prim;
    for (int d = 0; d < 3; ++d) { m.mom[d] = mom[d]; m.vel[d] = vel[d]; }
    m.cells = (int64_t)n[0] * n[1] * n[2];
    rc = alloc_member(b, m);
    if (rc) return rc;
    if (init) {
        // InitConsVarStag prob_type 1 (compressible_functions_stag.cpp:36-56), then
        // conservedToPrimitiveStag and FillBoundary as main_driver does
        const double rho0 = init[0], T0 = init[1];
        double cvmix = 0., e0mix = 0., rhoY[FHD_MAX_SPECIES];
        for (int i = 0; i < p.nspecies; ++i) {
            cvmix += init[2 + i] * p.hcv[i];
            e0mix += init[2 + i] * p.e0[i];
            rhoY[i] = rho0 * init[2 + i];
        }
        const double intEnergy = e0mix + T0 * cvmix;
        rc = init_uniform(cu, p.nspecies, rho0, rho0 * intEnergy, rhoY, b->stream);
        for (int d = 0; d < 3 && !rc; ++d)
            rc = cuda_ok(cudaMemsetAsync(mom[d].data, 0, (size_t)pts(mom[d]) * sizeof(double), b->stream));
        if (!rc) rc = exact_convert(dev_params(p, dt, 0), prim, vel, cu, mom, nullptr, b->stream);
        if (!rc) {
            GhostReq g[5] = {{cu, 0, 5 + p.nspecies}, {prim, 0, 6 + 2 * p.nspecies}, {vel[0], 0, 1}, {vel[1], 0, 1},
                             {vel[2], 0, 1}};
            rc = fill_ghosts(g, 5, n, b->stream);
        }
        if (rc) {
            cudaFreeAsync(m.scratch, b->stream);
            return rc;
        }
    }
    b->mode = mode;
    b->mem.push_back(m);
    b->dirty = true;
    *member = m.id;
    return FHD_OK;
}

int fhd_batch_remove(fhd_batch* b, int member) {
    if (!b) return FHD_ERR_BAD_ARG;
    const int q = find(b, member);
    if (q < 0) return FHD_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    int rc = sync_steps(b);
    if (rc) return rc;
    cudaFreeAsync(b->mem[q].scratch, b->stream);
    b->mem.erase(b->mem.begin() + q);
    b->dirty = true;
    return FHD_OK;
}

int fhd_batch_step(fhd_batch* b, int nsteps, int use_graph) {
    if (!b || nsteps < 0) return FHD_ERR_BAD_ARG;
    if (b->mem.empty() || nsteps == 0) return FHD_OK;
    cudaSetDevice(b->device);
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    if (!use_graph) {
        for (int s = 0; s < nsteps; ++s) {
            int rc = run_plan(b);
            if (rc) return rc;
        }
        return FHD_OK;
    }
    if (!b->gexec) {
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return cuda_ok(cudaGetLastError());
        int rc = run_plan(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc ? rc : FHD_ERR_CUDA;
        }
        b->graph = g;
        if (cudaGraphInstantiate(&b->gexec, g, 0) != cudaSuccess) {
            drop_graph(b);
            return cuda_ok(cudaGetLastError());
        }
    }
    for (int s = 0; s < nsteps; ++s)
        if (cudaGraphLaunch(b->gexec, b->stream) != cudaSuccess) return cuda_ok(cudaGetLastError());
    return FHD_OK;
}

int fhd_batch_size(const fhd_batch* b) { return b ? (int)b->mem.size() : -1; }

int fhd_batch_set_persistent(fhd_batch* b, int enable, int tile) {
    if (!b || tile < -1 || tile >= batch_face_tiles()) return FHD_ERR_BAD_ARG;
    if ((enable != 0) != b->persistent || tile != b->persist_tile) {
        b->persistent = enable != 0;
        b->persist_tile = tile;
        drop_graph(b);
    }
    return FHD_OK;
}

int fhd_batch_set_wait_limit(fhd_batch* b, double seconds, int hold_phase) {
    if (!b || !(seconds > 0) || seconds > 60 || hold_phase < -1 || hold_phase >= 24) return FHD_ERR_BAD_ARG;
    b->wait_limit_s = seconds;
    b->hold_phase = hold_phase;
    b->pargs.limit_ns = (unsigned long long)(seconds * 1e9);
    b->pargs.hold_phase = hold_phase;
    drop_graph(b);
    return FHD_OK;
}

int fhd_batch_num_tiles(void) { return batch_face_tiles(); }

int fhd_batch_set_tile(fhd_batch* b, int tile) {
    if (!b || tile < -1 || tile >= batch_face_tiles()) return FHD_ERR_BAD_ARG;
    if (tile != b->tile) {
        b->tile = tile;
        drop_graph(b);
    }
    return FHD_OK;
}

int fhd_batch_autotune(fhd_batch* b, int reps, double* ms, int* best) {
    if (!b || reps < 1) return FHD_ERR_BAD_ARG;
    if (b->mem.empty()) {
        if (best) *best = b->tile;
        return FHD_OK;
    }
    cudaSetDevice(b->device);
    if (b->dirty) {
        const int rc = rebuild(b);
        if (rc) return rc;
    }
    std::vector<const Launch*> faces;  // the face launches of the first stage
    for (const Launch& L : b->plan)
        if (L.kind >= 2 && L.kind <= 4 && faces.size() < 3) faces.push_back(&L);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return cuda_ok(cudaGetLastError());
    }
    char* d = static_cast<char*>(b->dbuf);
    const int nt = batch_face_tiles();
    int bt = b->tile, rc = FHD_OK;
    double bms = 0.0;
    for (int t = 0; t < nt && !rc; ++t) {
        for (int r = 0; r <= reps && !rc; ++r) {
            if (r == 1 && cudaEventRecord(e0, b->stream) != cudaSuccess) rc = FHD_ERR_CUDA;
            for (const Launch* L : faces)
                if (!rc)
                    rc = batch_launch(b->ns, b->mixed, L->kind, b->mode, t, d + L->args_off,
                                      reinterpret_cast<const int*>(d + L->bpref_off), L->nitems, L->nblocks, b->stream);
        }
        float el = 0.f;
        if (!rc && (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&el, e0, e1) != cudaSuccess))
            rc = FHD_ERR_CUDA;
        if (rc) break;
        const double per = (double)el / reps;
        if (ms) ms[t] = per;
        if (t == 0 || per < bms) {
            bms = per;
            bt = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        cudaGetLastError();
        return rc;
    }
    if (bt != b->tile) {
        b->tile = bt;
        drop_graph(b);
    }
    if (best) *best = bt;
    return FHD_OK;
}

int fhd_batch_member_status(fhd_batch* b, int member) {
    if (!b) return FHD_ERR_BAD_ARG;
    const int q = find(b, member);
    if (q < 0) return FHD_ERR_BAD_ARG;
    if (b->dirty || !b->dstatus) return FHD_OK;  // not stepped since it joined
    int h = 0;
    if (cudaMemcpyAsync(&h, b->dstatus + q, sizeof(int), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return cuda_ok(cudaGetLastError());
    return h;
}

int fhd_batch_synchronize(fhd_batch* b) {
    if (!b) return FHD_ERR_BAD_ARG;
    return cuda_ok(cudaStreamSynchronize(b->stream));
}

}  // extern "C"
