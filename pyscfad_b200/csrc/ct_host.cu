// Host orchestration and the extern "C" boundary of the B200 CCSD(T) library.
//
// Job planning replaces _ccsd_t_gen_jobs (pyscfadlib/.../vjp/cc/ccsd_t.c:6-72)
// and the Python slab loop (pyscfad/cc/ccsd_t.py:135-177): the sorted triples
// a>=b>=c are grouped into virtual super-blocks (A>=B>=C blocks of size Tv) so
// that one wave's terms share few t2T slabs, and super-blocks are packed into
// waves whose scratch (7 o^3 values per job) stays within a fixed budget.
// The per-thread private gradient copies + omp_dsum_reduce_inplace of the
// reference (ccsd_t_vjp.c:379-493, omp_reduce.c:6-24) become on-device
// accumulation into the caller's gradient buffers.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "ct_mixed.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {

#define CT_CK(call)                                                                  \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess) {                                                     \
            if (std::getenv("CTB_DEBUG"))                                            \
                std::fprintf(stderr, "ctb: %s failed: %s (%s:%d)\n", #call,          \
                             cudaGetErrorString(_e), __FILE__, __LINE__);            \
            return (_e == cudaErrorMemoryAllocation) ? CT_ERR_NOMEM : CT_ERR_CUDA;   \
        }                                                                            \
    } while (0)

cudaError_t smem_optin(const void *kernel, int bytes) {
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> done;   // (kernel, device) with the limit raised
    static std::vector<int> done_bytes;
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < done.size(); ++i)
        if (done[i].first == kernel && done[i].second == dev && done_bytes[i] >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    done.push_back({kernel, dev});
    done_bytes.push_back(bytes);
    return cudaSuccess;
}

struct Plan {
    int o = 0, v = 0, max_wave = 0;
    std::vector<int> jobs, wave_begin, tb_entries, tb_groups, tb_group_begin;
    std::vector<int> zchunks, zchunk_begin, x_entries, xgroups, xgroup_begin, xchunks, xchunk_begin;
    std::vector<int> ochunks, ochunk_begin;
    int *d_jobs = nullptr, *d_tb_entries = nullptr, *d_tb_groups = nullptr;
    int *d_zchunks = nullptr, *d_x_entries = nullptr, *d_xgroups = nullptr, *d_xchunks = nullptr;
    int *d_ochunks = nullptr;
    int n_waves() const { return (int)wave_begin.size() - 1; }
    void free_dev() {
        if (d_jobs) cudaFree(d_jobs);
        if (d_tb_entries) cudaFree(d_tb_entries);
        if (d_tb_groups) cudaFree(d_tb_groups);
        for (int *q : {d_zchunks, d_x_entries, d_xgroups, d_xchunks, d_ochunks})
            if (q) cudaFree(q);
        d_jobs = d_tb_entries = d_tb_groups = nullptr;
        d_zchunks = d_x_entries = d_xgroups = d_xchunks = d_ochunks = nullptr;
    }
};

// Fill waves/TB groups of a plan from super-blocks (each a list of jobs).
static void finish_plan(Plan &P, const std::vector<std::vector<int>> &blocks) {
    P.jobs.clear();
    P.wave_begin.assign(1, 0);
    const size_t mw = (size_t)P.max_wave;
    for (const auto &blk : blocks) {
        // waves are filled to max_wave: a super-block that does not fit is
        // continued in the next wave (the order keeps neighbours together)
        for (size_t pos = 0; pos < blk.size();) {
            const size_t room = mw - (P.jobs.size() - (size_t)P.wave_begin.back());
            const size_t take = std::min(room, blk.size() - pos);
            P.jobs.insert(P.jobs.end(), blk.begin() + pos, blk.begin() + pos + take);
            pos += take;
            if (P.jobs.size() - (size_t)P.wave_begin.back() == mw) P.wave_begin.push_back((int)P.jobs.size());
        }
    }
    if ((int)P.jobs.size() > P.wave_begin.back()) P.wave_begin.push_back((int)P.jobs.size());
    // K_TB groups: per wave, term ids sorted by z
    P.tb_entries.clear();
    P.tb_groups.clear();
    P.tb_group_begin.assign(1, 0);
    std::vector<int> cnt(P.v + 1);
    for (int w = 0; w < P.n_waves(); ++w) {
        const int j0 = P.wave_begin[w], j1 = P.wave_begin[w + 1];
        std::fill(cnt.begin(), cnt.end(), 0);
        for (int j = j0; j < j1; ++j) {
            int a, b, c;
            unpack_job(P.jobs[j], a, b, c);
            for (int s = 0; s < 6; ++s) {
                int x, y, z;
                term_xyz(s, a, b, c, x, y, z);
                cnt[z + 1]++;
            }
        }
        for (int z = 0; z < P.v; ++z) cnt[z + 1] += cnt[z];
        const int base = (int)P.tb_entries.size();
        P.tb_entries.resize(base + 6 * (j1 - j0));
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int j = j0; j < j1; ++j) {
            int a, b, c;
            unpack_job(P.jobs[j], a, b, c);
            for (int s = 0; s < 6; ++s) {
                int x, y, z;
                term_xyz(s, a, b, c, x, y, z);
                P.tb_entries[base + fill[z]++] = (j - j0) * 6 + s;
            }
        }
        for (int z = 0; z < P.v; ++z)
            if (cnt[z + 1] > cnt[z]) {
                P.tb_groups.push_back(z);
                P.tb_groups.push_back(base + cnt[z]);
                P.tb_groups.push_back(base + cnt[z + 1]);
            }
        P.tb_group_begin.push_back((int)P.tb_groups.size() / 3);
    }
    // mixed-path tables: z-groups cut into chunks of <= nt_z terms; x-sorted
    // terms with their groups, chunks of <= nt_x terms (F2: each term takes
    // ceil(o / 64) * 64 accumulator columns, the bf16 row width, which the tf32
    // width 32 divides) and chunks of <= nt_z terms (OB2: o columns per term);
    // 256 columns at most
    const int o64 = (P.o + 63) / 64 * 64;
    const int nt_z = std::max(1, std::min(32, 256 / std::max(1, P.o)));
    const int nt_x = std::max(1, 256 / o64);
    P.zchunks.clear(); P.zchunk_begin.assign(1, 0);
    P.x_entries.clear(); P.xgroups.clear(); P.xgroup_begin.assign(1, 0);
    P.xchunks.clear(); P.xchunk_begin.assign(1, 0);
    P.ochunks.clear(); P.ochunk_begin.assign(1, 0);
    for (int w = 0; w < P.n_waves(); ++w) {
        for (int g = P.tb_group_begin[w]; g < P.tb_group_begin[w + 1]; ++g) {
            const int z = P.tb_groups[3 * g], e0 = P.tb_groups[3 * g + 1], e1 = P.tb_groups[3 * g + 2];
            for (int e = e0; e < e1; e += nt_z) {
                P.zchunks.push_back(z);
                P.zchunks.push_back(e);
                P.zchunks.push_back(std::min(e1, e + nt_z));
            }
        }
        P.zchunk_begin.push_back((int)P.zchunks.size() / 3);
        const int j0 = P.wave_begin[w], j1 = P.wave_begin[w + 1];
        std::fill(cnt.begin(), cnt.end(), 0);
        for (int j = j0; j < j1; ++j) {
            int a, b, c;
            unpack_job(P.jobs[j], a, b, c);
            for (int s = 0; s < 6; ++s) {
                int x, y, z;
                term_xyz(s, a, b, c, x, y, z);
                cnt[x + 1]++;
            }
        }
        for (int x = 0; x < P.v; ++x) cnt[x + 1] += cnt[x];
        const int base = (int)P.x_entries.size();
        P.x_entries.resize(base + 6 * (j1 - j0));
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int j = j0; j < j1; ++j) {
            int a, b, c;
            unpack_job(P.jobs[j], a, b, c);
            for (int s = 0; s < 6; ++s) {
                int x, y, z;
                term_xyz(s, a, b, c, x, y, z);
                P.x_entries[base + fill[x]++] = (j - j0) * 6 + s;
            }
        }
        for (int x = 0; x < P.v; ++x)
            if (cnt[x + 1] > cnt[x]) {
                const int e0 = base + cnt[x], e1 = base + cnt[x + 1];
                P.xgroups.push_back(x); P.xgroups.push_back(e0); P.xgroups.push_back(e1);
                for (int e = e0; e < e1; e += nt_x) {
                    P.xchunks.push_back(x);
                    P.xchunks.push_back(e);
                    P.xchunks.push_back(std::min(e1, e + nt_x));
                }
                for (int e = e0; e < e1; e += nt_z) {
                    P.ochunks.push_back(x);
                    P.ochunks.push_back(e);
                    P.ochunks.push_back(std::min(e1, e + nt_z));
                }
            }
        P.xgroup_begin.push_back((int)P.xgroups.size() / 3);
        P.xchunk_begin.push_back((int)P.xchunks.size() / 3);
        P.ochunk_begin.push_back((int)P.ochunks.size() / 3);
    }
}

static int upload_plan(Plan &P) {
    P.free_dev();
    CT_CK(cudaMalloc(&P.d_jobs, std::max<size_t>(1, P.jobs.size()) * sizeof(int)));
    CT_CK(cudaMalloc(&P.d_tb_entries, std::max<size_t>(1, P.tb_entries.size()) * sizeof(int)));
    CT_CK(cudaMalloc(&P.d_tb_groups, std::max<size_t>(1, P.tb_groups.size()) * sizeof(int)));
    CT_CK(cudaMemcpy(P.d_jobs, P.jobs.data(), P.jobs.size() * sizeof(int), cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(P.d_tb_entries, P.tb_entries.data(), P.tb_entries.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(P.d_tb_groups, P.tb_groups.data(), P.tb_groups.size() * sizeof(int),
                     cudaMemcpyHostToDevice));
    auto up = [](int **d, const std::vector<int> &h) -> cudaError_t {
        cudaError_t e = cudaMalloc(d, std::max<size_t>(1, h.size()) * sizeof(int));
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice);
    };
    CT_CK(up(&P.d_zchunks, P.zchunks));
    CT_CK(up(&P.d_x_entries, P.x_entries));
    CT_CK(up(&P.d_xgroups, P.xgroups));
    CT_CK(up(&P.d_xchunks, P.xchunks));
    CT_CK(up(&P.d_ochunks, P.ochunks));
    return CT_OK;
}

// all sorted jobs, virtual super-block order
static void plan_full(Plan &P) {
    int tv = std::max(1, (int)std::floor(std::cbrt((double)P.max_wave) + 1e-9));
    tv = std::min(tv, P.v);
    const int nb = (P.v + tv - 1) / tv;
    std::vector<std::vector<int>> blocks;
    for (int A = 0; A < nb; ++A)
        for (int B = 0; B <= A; ++B)
            for (int C = 0; C <= B; ++C) {
                std::vector<int> blk;
                for (int a = A * tv; a < std::min(P.v, (A + 1) * tv); ++a)
                    for (int b = B * tv; b < std::min(a + 1, (B + 1) * tv); ++b)
                        for (int c = C * tv; c < std::min(b + 1, (C + 1) * tv); ++c)
                            blk.push_back(pack_job(a, b, c));
                if (!blk.empty()) blocks.push_back(std::move(blk));
            }
    finish_plan(P, blocks);
}

// Orders a set of sorted jobs (packed) into virtual super-blocks of side
// ~cbrt(wave): the jobs of a wave then share few distinct x, y and z, so the
// tensor-core kinds grouped by z (t2-bar) or x (vooo-bar) get long K loops and
// few output tiles, and the vvop/t2T slabs a wave reads stay in L2.  Appends
// one list per super-block to blocks.
static void grouped_blocks(const Plan &P, const std::vector<int> &packed, std::vector<std::vector<int>> &blocks) {
    int tv = std::max(1, (int)std::floor(std::cbrt((double)P.max_wave) + 1e-9));
    tv = std::min(tv, P.v);
    const long long nb = (P.v + tv - 1) / tv;
    std::vector<std::pair<long long, int>> keyed(packed.size());
    for (size_t t = 0; t < packed.size(); ++t) {
        int a, b, c;
        unpack_job(packed[t], a, b, c);
        keyed[t] = {((long long)(a / tv) * nb + b / tv) * nb + c / tv, packed[t]};
    }
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<long long, int> &x, const std::pair<long long, int> &y) {
                         return x.first < y.first;
                     });
    long long cur = -1;
    for (const auto &kv : keyed) {
        if (kv.first != cur) { blocks.emplace_back(); cur = kv.first; }
        blocks.back().push_back(kv.second);
    }
}

static void plan_grouped(Plan &P, const std::vector<int> &packed) {
    std::vector<std::vector<int>> blocks;
    grouped_blocks(P, packed, blocks);
    finish_plan(P, blocks);
}

// The jobs of one reference slab block (a0, a1, b0, b1), as _ccsd_t_gen_jobs
// enumerates them (ccsd_t.c:16-69), split into stages by their smallest index
// c: stage 0 the jobs with c >= b0 (all their indices lie in the slabs),
// stage k >= 1 those with c in [(k-1) cw, min(k cw, b0)), cw chosen so that
// a stage (every slab pair (a, b) times cw values of c) is about one wave of
// max_wave jobs.  Such a stage touches few distinct rows (the slabs' and cw
// others), where super-blocks of a block whose slabs are narrow span almost
// every c in each wave.  Returns the number of stages; rows(k) of a stage:
// [b0, a1) for stage 0, its c range otherwise.
static int block_stages(int a0, int a1, int b0, int b1, int max_wave, int *cw_out,
                        std::vector<std::vector<int>> &sjobs) {
    const bool diag = b0 == a0 && b1 == a1;
    const long long npair = diag ? (long long)(a1 - a0) * (a1 - a0 + 1) / 2 : (long long)(a1 - a0) * (b1 - b0);
    const int cw = (int)std::max<long long>(1, max_wave / npair);
    const int S = 1 + (b0 + cw - 1) / cw;
    sjobs.assign(S, {});
    for (int a = a0; a < a1; ++a)
        for (int b = diag ? a0 : b0; b < (diag ? a + 1 : b1); ++b)
            for (int c = 0; c <= b; ++c) sjobs[c >= b0 ? 0 : 1 + c / cw].push_back(pack_job(a, b, c));
    *cw_out = cw;
    return S;
}

// one reference slab block: its stages in order, super-blocks within each
static void plan_block(Plan &P, int a0, int a1, int b0, int b1) {
    std::vector<std::vector<int>> sjobs, blocks;
    int cw = 1;
    block_stages(a0, a1, b0, b1, P.max_wave, &cw, sjobs);
    for (const auto &j : sjobs) grouped_blocks(P, j, blocks);
    finish_plan(P, blocks);
}

// jobs a0 <= a < a1, all b <= a, c <= b (lnoccsdt_contract's a-slab, lno_ccsd_t.c:73-94 folded
// onto sorted triples)
static void plan_aslab(Plan &P, int a0, int a1) {
    std::vector<int> jobs;
    for (int a = a0; a < a1; ++a)
        for (int b = 0; b <= a; ++b)
            for (int c = 0; c <= b; ++c) jobs.push_back(pack_job(a, b, c));
    plan_grouped(P, jobs);
}

// an explicit list of sorted jobs (host triples a >= b >= c)
static void plan_list(Plan &P, const int *abc, int njobs) {
    std::vector<int> jobs((size_t)njobs);
    for (int t = 0; t < njobs; ++t) jobs[t] = pack_job(abc[3 * t], abc[3 * t + 1], abc[3 * t + 2]);
    plan_grouped(P, jobs);
}

// Device and pinned host buffers of the host-pointer entry, kept across calls
// (grown when needed; freed by ct_release_workspace): allocating and faulting in
// tens of GB per call would cost more than the call's copies.
struct HostPathCache {
    enum { MO, T1, T2, VOOO, FVO, VVOP, NBUF };
    double *in[NBUF] = {}, *bar[NBUF] = {};
    size_t in_cap[NBUF] = {}, bar_cap[NBUF] = {};
    double *pin = nullptr;   // pinned staging ring for device -> host gradient reads (2 halves)
    size_t pin_cap = 0;
    cudaStream_t st = nullptr;       // the host path's own stream (device work)
    cudaStream_t st_in = nullptr;    // copies in, one stage ahead of the device work
    cudaStream_t st_out = nullptr;   // gradients out of finished stages
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void release() {
        for (int i = 0; i < NBUF; ++i) {
            if (in[i]) cudaFree(in[i]);
            if (bar[i]) cudaFree(bar[i]);
            in[i] = bar[i] = nullptr;
            in_cap[i] = bar_cap[i] = 0;
        }
        if (pin) cudaFreeHost(pin);
        pin = nullptr;
        pin_cap = 0;
        for (auto &e : ev)
            if (e) { cudaEventDestroy(e); e = nullptr; }
        if (st) { cudaStreamDestroy(st); st = nullptr; }
        if (st_in) { cudaStreamDestroy(st_in); st_in = nullptr; }
        if (st_out) { cudaStreamDestroy(st_out); st_out = nullptr; }
    }
};
// Optional per-kernel timing: CUDA events around each launch on the launch
// stream, summed per kernel kind when read back.
struct Prof {
    bool on = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[kProfKinds];
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        cudaEvent_t e;
        if (!pool.empty()) { e = pool.back(); pool.pop_back(); }
        else cudaEventCreate(&e);
        return e;
    }
    void clear() {
        for (auto &v : ev) {
            for (auto &p : v) { pool.push_back(p.first); pool.push_back(p.second); }
            v.clear();
        }
    }
};
constexpr int kMaxDevices = 64;

// Everything the library keeps between calls on one device: cached plans,
// wave scratch, per-job energies, the host-pointer path's buffers and the
// profiling events.  Device memory belongs to the device it was allocated on,
// so each device has its own workspace, selected by the device current at
// the call; its mutex serializes calls on that device.
struct Workspace {
    std::mutex mu;
    Plan full;                       // cached plan of the last full problem
    Plan block;                      // cached plan of the last block call
    int block_key[7] = {-1, -1, -1, -1, -1, -1, -1};
    size_t scratch_bytes = 0;
    void *scratch = nullptr;
    long long job_e_n = 0;
    double *job_e = nullptr;
    int orb_o = -1;
    int *orbits = nullptr;
    int n_orb = 0;
    double *e_tmp = nullptr;
    double *red_work = nullptr;     // 2 * kReduceParts partial sums
    HostPathCache hp;
    Prof prof;
    cudaEvent_t prof_open[kProfKinds] = {};
    int cc_major = -1;              // compute capability major, read once
    int sm_count = 0;
    double budget_mb = -1.0;        // wave scratch budget, fixed at the first call
    void release() {
        full.free_dev();
        full = Plan();
        block.free_dev();
        block = Plan();
        for (int &k : block_key) k = -1;
        if (scratch) cudaFree(scratch);
        if (job_e) cudaFree(job_e);
        if (orbits) cudaFree(orbits);
        if (e_tmp) cudaFree(e_tmp);
        if (red_work) cudaFree(red_work);
        scratch = nullptr; job_e = nullptr; orbits = nullptr; e_tmp = nullptr; red_work = nullptr;
        scratch_bytes = 0; job_e_n = 0; orb_o = -1; n_orb = 0;
        hp.release();
    }
};
static Workspace g_ws[kMaxDevices];

// The current device's workspace after checking that it is an sm_100 part
// (the check is made once per device); null with *rc set otherwise.
static Workspace *device_ws(int *rc) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *rc = CT_ERR_NO_DEVICE;
        return nullptr;
    }
    Workspace &W = g_ws[dev];
    std::lock_guard<std::mutex> lk(W.mu);
    if (W.cc_major < 0) {
        int major = 0, sms = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            *rc = CT_ERR_NO_DEVICE;
            return nullptr;
        }
        W.cc_major = major;
        W.sm_count = sms;
    }
    if (W.cc_major != 10) {
        *rc = CT_ERR_NO_DEVICE;
        return nullptr;
    }
    *rc = CT_OK;
    return &W;
}

// the current device's workspace without the architecture check (profiling
// and size queries); null when no device ordinal is current
static Workspace *current_ws() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    return &g_ws[dev];
}


struct ProfScope {
    Prof &pr; int kind; cudaStream_t st; cudaEvent_t b{}, e{};
    ProfScope(Prof &p, int k, cudaStream_t s) : pr(p), kind(k), st(s) {
        if (pr.on) { b = pr.get(); cudaEventRecord(b, st); }
    }
    ~ProfScope() {
        if (pr.on) { e = pr.get(); cudaEventRecord(e, st); pr.ev[kind].push_back({b, e}); }
    }
};
#define CT_PROF(kind) ProfScope _ps_##__LINE__(W.prof, (kind), st)

// begin/end callback used by the mixed path
struct ProfCtx {
    Workspace *W;
    cudaStream_t st;
};
static int prof_cb(int kind, int end, void *ctx) {
    ProfCtx *c = static_cast<ProfCtx *>(ctx);
    cudaEvent_t e = c->W->prof.get();
    cudaEventRecord(e, c->st);
    if (!end) c->W->prof_open[kind] = e;
    else c->W->prof.ev[kind].push_back({c->W->prof_open[kind], e});
    return 0;
}

static long long n_sorted(long long v) { return v * (v + 1) * (v + 2) / 6; }

static size_t scratch_elt(int mode) { return mode == CT_MODE_FP64 ? sizeof(double) : sizeof(float); }

// Scratch budget of a device's wave buffers, fixed at its first call:
// CTB_SCRATCH_MB if set, else 16 GiB or a quarter of the then free device
// memory, whichever is smaller (at least 256 MiB).
static double scratch_budget_mb(Workspace &W) {
    if (W.budget_mb < 0.0) {
        double mb;
        if (const char *s = std::getenv("CTB_SCRATCH_MB")) {
            mb = std::atof(s);
        } else {
            size_t fr = 0, tot = 0;
            mb = 16384.0;   // 16 GiB: 1.713 s vs 1.726 s (8 GiB) and 1.779 s (4 GiB) per nocc=48/nvir=500 step
            if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) mb = std::min(mb, 0.25 * (double)fr / 1048576.0);
            mb = std::max(mb, 256.0);
        }
        W.budget_mb = mb;
    }
    return W.budget_mb;
}

// Jobs per wave: as many as the scratch budget holds (at most 8192), rounded
// down to a multiple of two CTAs per SM so the per-job kernels fill whole
// rounds of the GPU.
static int max_wave_jobs(Workspace &W, int o, int mode) {
    const double per_job = (double)kSlots * o * o * o * scratch_elt(mode)
                         + (mode == CT_MODE_FP64 ? 0.0 : mixed_extra_bytes_per_job(o, mode));
    long long mw = (long long)(scratch_budget_mb(W) * 1048576.0 / per_job);
    mw = std::max<long long>(1, std::min<long long>(mw, 8192));
    const long long round = 2LL * (W.sm_count > 0 ? W.sm_count : 148);
    if (mw >= round) mw -= mw % round;
    if (const char *s = std::getenv("CTB_MAX_WAVE")) mw = std::max(1, std::atoi(s));
    return (int)mw;
}

static int ensure_common(Workspace &W, int o, int v, int mode, int max_wave) {
    const size_t need = (size_t)max_wave * kSlots * (size_t)o * o * o * scratch_elt(mode)
                      + (mode == CT_MODE_FP64 ? 0 : (size_t)(max_wave * mixed_extra_bytes_per_job(o, mode)));
    if (need > W.scratch_bytes) {
        if (W.scratch) cudaFree(W.scratch);
        W.scratch = nullptr;
        W.scratch_bytes = 0;
        CT_CK(cudaMalloc(&W.scratch, need));
        W.scratch_bytes = need;
    }
    const long long nj = n_sorted(v);
    if (nj > W.job_e_n) {
        if (W.job_e) cudaFree(W.job_e);
        W.job_e = nullptr;
        W.job_e_n = 0;
        CT_CK(cudaMalloc(&W.job_e, nj * sizeof(double)));
        W.job_e_n = nj;
    }
    if (W.orb_o != o) {
        std::vector<int> orb;
        for (int i = 0; i < o; ++i)
            for (int j = 0; j <= i; ++j)
                for (int k = 0; k <= j; ++k) orb.push_back(i | (j << 8) | (k << 16));
        if (W.orbits) cudaFree(W.orbits);
        W.orbits = nullptr;
        CT_CK(cudaMalloc(&W.orbits, orb.size() * sizeof(int)));
        CT_CK(cudaMemcpy(W.orbits, orb.data(), orb.size() * sizeof(int), cudaMemcpyHostToDevice));
        W.orb_o = o;
        W.n_orb = (int)orb.size();
    }
    if (!W.e_tmp) CT_CK(cudaMalloc(&W.e_tmp, sizeof(double)));
    if (!W.red_work) CT_CK(cudaMalloc(&W.red_work, 2 * kReduceParts * sizeof(double)));
    return CT_OK;
}

static int validate(const ct_problem *p, int mode) {
    if (!p) return CT_ERR_NULL;
    if (p->nocc < 1 || p->nocc > 255 || p->nvir < 1 || p->nvir > 1024) return CT_ERR_SHAPE;
    if (!p->mo_energy || !p->t1T || !p->t2T || !p->vooo || !p->fvo || !p->vvop) return CT_ERR_NULL;
    if (mode != CT_MODE_FP64 && mode != CT_MODE_TF32 && mode != CT_MODE_BF16X3) return CT_ERR_MODE;
    return CT_OK;
}

// LNO-projected selection: projector (device, o x o); orderings (x, y, z)
// with x in [a0, a1), y in [b0, b1), z in [c0, c1); for the VJP, mat_bar
// (device, o x o, accumulates) and part (max_wave x o x o doubles of scratch)
struct LnoSel {
    const double *mat = nullptr;
    int a0 = 0, a1 = 0, b0 = 0, b1 = 0, c0 = 0, c1 = 0;
    double *mat_bar = nullptr, *part = nullptr;
};

// Kernel arguments of one call (LNO selection, inputs, gradients, tables).
static EpiArgs epi_args(Workspace &W, const ct_problem *p, bool vjp, double et_bar, const ct_grads *g,
                        double *job_e, const LnoSel *lno, double *t3_c = nullptr, double *t3_x = nullptr) {
    const int o = p->nocc, v = p->nvir, n = o + v;
    EpiArgs ea{};
    if (lno) {
        ea.lno_mat = lno->mat;
        ea.lno_a0 = lno->a0; ea.lno_a1 = lno->a1;
        ea.lno_b0 = lno->b0; ea.lno_b1 = lno->b1;
        ea.lno_c0 = lno->c0; ea.lno_c1 = lno->c1;
        ea.lno_phase = vjp ? 2 : 1;
        ea.lno_mat_bar_part = lno->part;
    }
    ea.o = o; ea.v = v; ea.n = n;
    ea.mo_energy = p->mo_energy; ea.t1T = p->t1T; ea.t2T = p->t2T; ea.fvo = p->fvo; ea.vvop = p->vvop;
    ea.et_bar = et_bar;
    ea.with_vjp = vjp ? 1 : 0;
    ea.job_e = job_e;
    if (vjp) {
        ea.mo_energy_bar = g->mo_energy; ea.t1T_bar = g->t1T; ea.t2T_bar = g->t2T;
        ea.fvo_bar = g->fvo; ea.vvop_bar = g->vvop;
    }
    ea.orbits = W.orbits;
    ea.n_orb = W.n_orb;
    ea.t3_c = t3_c;
    ea.t3_x = t3_x;
    return ea;
}

// Every wave of plan P on stream st, the mixed path with operands mo
// already converted for the rows P's jobs read.
static int run_waves(Workspace &W, const Plan &P, const ct_problem *p, int mode, bool vjp, const ct_grads *g,
                     const EpiArgs &ea, const MixedOperands &mo, double *lno_mat_bar, cudaStream_t st) {
    const int o = p->nocc, v = p->nvir, n = o + v;
    const double *lno_mat = ea.lno_mat;
    for (int w = 0; w < P.n_waves(); ++w) {
        WaveView wv{};
        wv.o = o; wv.v = v; wv.n = n;
        wv.n_jobs = P.wave_begin[w + 1] - P.wave_begin[w];
        wv.jobs = P.d_jobs + P.wave_begin[w];
        wv.n_tb_groups = P.tb_group_begin[w + 1] - P.tb_group_begin[w];
        wv.tb_entries = P.d_tb_entries;
        wv.tb_groups = P.d_tb_groups + 3 * P.tb_group_begin[w];
        wv.n_zchunks = P.zchunk_begin[w + 1] - P.zchunk_begin[w];
        wv.zchunks = P.d_zchunks + 3 * P.zchunk_begin[w];
        wv.x_entries = P.d_x_entries;
        wv.n_xgroups = P.xgroup_begin[w + 1] - P.xgroup_begin[w];
        wv.xgroups = P.d_xgroups + 3 * P.xgroup_begin[w];
        wv.n_xchunks = P.xchunk_begin[w + 1] - P.xchunk_begin[w];
        wv.xchunks = P.d_xchunks + 3 * P.xchunk_begin[w];
        wv.n_ochunks = P.ochunk_begin[w + 1] - P.ochunk_begin[w];
        wv.ochunks = P.d_ochunks + 3 * P.ochunk_begin[w];
        if (mode == CT_MODE_FP64) {
            double *S = (double *)W.scratch;
            { CT_PROF(PK_F1); CT_CK(f64_gemm(K_F1, wv, p->t2T, p->vvop, S, S, st)); }
            { CT_PROF(PK_F2); CT_CK(f64_gemm(K_F2, wv, p->vooo, p->t2T, S, S, st)); }
            if (lno_mat && vjp) {
                // LNO VJP: forward pass (W, z/D cubes), projections A, B with the
                // energy and mat_bar partials, backward pass (W-bar, ybar), then
                // the canonical bars
                EpiArgs ef = ea;
                ef.with_vjp = 0;
                ef.lno_phase = 1;
                { CT_PROF(PK_EPI); CT_CK(f64_epilogue(wv, ef, S, st)); }
                { CT_PROF(PK_RED); CT_CK(f64_lno_vjp_project(wv, ea, S, st)); }
                { CT_PROF(PK_EPI); CT_CK(f64_epilogue(wv, ea, S, st)); }
                { CT_PROF(PK_RED); CT_CK(f64_lno_mat_bar(wv, ea, lno_mat_bar, st)); }
            } else {
                { CT_PROF(PK_EPI); CT_CK(f64_epilogue(wv, ea, S, st)); }
                if (lno_mat) { CT_PROF(PK_VT); CT_CK(f64_lno_contract(wv, ea, S, st)); }
            }
            if (vjp) {
                { CT_PROF(PK_VT); CT_CK(f64_vterm(wv, ea, S, st)); }
                { CT_PROF(PK_VB); CT_CK(f64_gemm(K_VB, wv, p->t2T, S, g->vvop, S, st)); }
                { CT_PROF(PK_TB); CT_CK(f64_gemm(K_TB, wv, p->vvop, S, g->t2T, S, st)); }
                { CT_PROF(PK_OB1); CT_CK(f64_gemm(K_OB1, wv, S, p->t2T, g->vooo, S, st)); }
                { CT_PROF(PK_OB2); CT_CK(f64_gemm(K_OB2, wv, p->vooo, S, g->t2T, S, st)); }
            }
        } else {
            ProfCtx pc{&W, st};
            int rc = mixed_wave(wv, ea, p, g, mo, mode, vjp, W.scratch, st, W.prof.on ? prof_cb : nullptr, &pc);
            if (rc == CT_OK && lno_mat && vjp) {
                CT_PROF(PK_RED);
                if (f64_lno_mat_bar(wv, ea, lno_mat_bar, st) != cudaSuccess) rc = CT_ERR_CUDA;
            }
            if (rc != CT_OK) return rc;
        }
    }
    return CT_OK;
}

// Runs every wave of plan P.  job_e must hold n_sorted(v) doubles (zeroed here).
// LNO-projected selection: see LnoSel.  lno switches the job energies to the
// LNO-projected form (any mode); with vjp, et_bar is then the reference LNO
// kernel's cotangent as passed (not doubled).
static int run_plan(Workspace &W, const Plan &P, const ct_problem *p, int mode, bool vjp, double et_bar,
                    const ct_grads *g, double *job_e, double *e_out, cudaStream_t st,
                    const LnoSel *lno = nullptr, double *t3_c = nullptr, double *t3_x = nullptr) {
    const int o = p->nocc, v = p->nvir;
    if (lno && (!lno->mat || o > 64 || (vjp && (!lno->mat_bar || !lno->part)))) return CT_ERR_MODE;
    if (t3_c && (mode != CT_MODE_FP64 || vjp || lno || !t3_x)) return CT_ERR_MODE;
    CT_CK(cudaMemsetAsync(job_e, 0, n_sorted(v) * sizeof(double), st));
    const EpiArgs ea = epi_args(W, p, vjp, et_bar, g, job_e, lno, t3_c, t3_x);
    MixedOperands mo{};
    if (mode != CT_MODE_FP64) {
        int rc = mixed_prepare(p, mode, &mo, st);
        if (rc != CT_OK) return rc;
    }
    int rc = run_waves(W, P, p, mode, vjp, g, ea, mo, lno ? lno->mat_bar : nullptr, st);
    if (mode != CT_MODE_FP64) {
        mixed_release(&mo, st);
        if (rc != CT_OK) return rc;
        rc = mixed_check_error(st);
    }
    if (rc != CT_OK) return rc;
    if (e_out) { CT_PROF(PK_RED); CT_CK(reduce_energy(job_e, n_sorted(v), e_out, W.red_work, st)); }
    return CT_OK;
}

// the cached plan of every sorted job (rebuilt when nocc, nvir or the wave size change)
static Plan *full_plan(Workspace &W, int o, int v, int mw, int *rc) {
    if (W.full.o != o || W.full.v != v || W.full.max_wave != mw || !W.full.d_jobs) {
        W.full.free_dev();
        W.full = Plan();
        W.full.o = o; W.full.v = v; W.full.max_wave = mw;
        plan_full(W.full);
        if ((*rc = upload_plan(W.full)) != CT_OK) { W.full.free_dev(); W.full = Plan(); return nullptr; }
    }
    *rc = CT_OK;
    return &W.full;
}

// kind: 0 = all jobs, 1 = reference slab block (a0,a1,b0,b1), 2 = a-slab [a0,a1)
static int run_sel(const ct_problem *p, int mode, bool vjp, double et_bar, const ct_grads *g,
                   double *e_out, double *job_e_out, cudaStream_t st, int kind, int a0, int a1, int b0,
                   int b1) {
    int rc = validate(p, mode);
    if (rc != CT_OK) return rc;
    if (vjp && (!g || !g->mo_energy || !g->t1T || !g->t2T || !g->vooo || !g->fvo || !g->vvop))
        return CT_ERR_NULL;
    const int v = p->nvir;
    if (kind == 1) {
        if (a0 < 0 || a1 > v || a0 >= a1 || b0 < 0 || b1 > a1 || b0 >= b1) return CT_ERR_SHAPE;
        if (!(b1 <= a0 || (b0 == a0 && b1 == a1))) return CT_ERR_SHAPE;
    } else if (kind == 2) {
        if (a0 < 0 || a1 > v || a0 >= a1) return CT_ERR_SHAPE;
    }
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    const int mw = max_wave_jobs(W, p->nocc, mode);
    if ((rc = ensure_common(W, p->nocc, p->nvir, mode, mw)) != CT_OK) return rc;
    Plan *P;
    if (kind == 0) {
        if (!(P = full_plan(W, p->nocc, v, mw, &rc))) return rc;
    } else {
        const int key[7] = {p->nocc, v, mw, kind, a0, a1, kind == 1 ? b0 * 4096 + b1 : 0};
        if (!W.block.d_jobs || !std::equal(key, key + 7, W.block_key)) {
            W.block.free_dev();
            W.block = Plan();
            W.block.o = p->nocc; W.block.v = v; W.block.max_wave = mw;
            if (kind == 1) plan_block(W.block, a0, a1, b0, b1);
            else plan_aslab(W.block, a0, a1);
            if ((rc = upload_plan(W.block)) != CT_OK) { W.block.free_dev(); W.block = Plan(); return rc; }
            std::copy(key, key + 7, W.block_key);
        }
        P = &W.block;
    }
    return run_plan(W, *P, p, mode, vjp, et_bar, g, job_e_out ? job_e_out : W.job_e, e_out, st);
}

// energy over an explicit job list (no VJP); the plan is rebuilt every call
static int run_list(const ct_problem *p, int mode, const int *abc, int njobs, double *e_out,
                    double *job_e_out, cudaStream_t st) {
    int rc = validate(p, mode);
    if (rc != CT_OK) return rc;
    if (!abc || njobs < 1) return njobs == 0 && abc ? CT_ERR_SHAPE : CT_ERR_NULL;
    const int v = p->nvir;
    if ((long long)njobs > n_sorted(v)) return CT_ERR_SHAPE;
    for (int t = 0; t < njobs; ++t) {
        const int a = abc[3 * t], b = abc[3 * t + 1], c = abc[3 * t + 2];
        if (!(a < v && a >= b && b >= c && c >= 0)) return CT_ERR_SHAPE;
    }
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    const int mw = max_wave_jobs(W, p->nocc, mode);
    if ((rc = ensure_common(W, p->nocc, v, mode, mw)) != CT_OK) return rc;
    W.block.free_dev();
    W.block = Plan();
    for (int &k : W.block_key) k = -1;
    W.block.o = p->nocc; W.block.v = v; W.block.max_wave = mw;
    plan_list(W.block, abc, njobs);
    if ((rc = upload_plan(W.block)) != CT_OK) { W.block.free_dev(); W.block = Plan(); return rc; }
    return run_plan(W, W.block, p, mode, false, 0.0, nullptr, job_e_out ? job_e_out : W.job_e, e_out, st);
}

// LNO-projected energy over the a-slab [a0, a1) of lnoccsdt_contract: every
// sorted job with a virtual index in the slab (its orderings with x outside
// the slab get weight 0 in the projection kernel).  Any precision mode.
static int run_lno(const ct_problem *p, int mode, const double *mat, int a0, int a1, double *e_out,
                   double *job_e_out, cudaStream_t st) {
    int rc = validate(p, mode);
    if (rc != CT_OK) return rc;
    if (!mat || (!e_out && !job_e_out)) return CT_ERR_NULL;
    const int v = p->nvir;
    if (p->nocc > 64 || a0 < 0 || a1 > v || a0 >= a1) return CT_ERR_SHAPE;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    const int mw = max_wave_jobs(W, p->nocc, mode);
    if ((rc = ensure_common(W, p->nocc, v, mode, mw)) != CT_OK) return rc;
    Plan *P;
    if (a0 == 0 && a1 == v) {
        // the whole range is every sorted job: the canonical path's cached plan
        if (!(P = full_plan(W, p->nocc, v, mw, &rc))) return rc;
    } else {
        // the sorted jobs with at least one index in the slab, cached by slab
        const int key[7] = {p->nocc, v, mw, 3, a0, a1, 0};
        if (!W.block.d_jobs || !std::equal(key, key + 7, W.block_key)) {
            std::vector<int> abc;
            for (int a = 0; a < v; ++a)
                for (int b = 0; b <= a; ++b)
                    for (int c = 0; c <= b; ++c)
                        if ((a >= a0 && a < a1) || (b >= a0 && b < a1) || (c >= a0 && c < a1)) {
                            abc.push_back(a); abc.push_back(b); abc.push_back(c);
                        }
            W.block.free_dev();
            W.block = Plan();
            for (int &k : W.block_key) k = -1;
            W.block.o = p->nocc; W.block.v = v; W.block.max_wave = mw;
            plan_list(W.block, abc.data(), (int)(abc.size() / 3));
            if ((rc = upload_plan(W.block)) != CT_OK) { W.block.free_dev(); W.block = Plan(); return rc; }
            std::copy(key, key + 7, W.block_key);
        }
        P = &W.block;
    }
    LnoSel sel;
    sel.mat = mat;
    sel.a0 = a0; sel.a1 = a1;
    sel.b0 = 0; sel.b1 = v; sel.c0 = 0; sel.c1 = v;
    return run_plan(W, *P, p, mode, false, 0.0, nullptr, job_e_out ? job_e_out : W.job_e, e_out, st, &sel);
}

static int run_lno_vjp_locked(Workspace &W, const ct_problem *p, int mode, const double *mat, double et_bar, int b0,
                              int b1, int c0, int c1, const ct_grads *g, double *mat_bar, double *e_out,
                              cudaStream_t st);

// LNO VJP over the slab block (b0, b1, c0, c1) of lnoccsdt_energy_vjp
// (lno_ccsd_t_vjp.c:355-398: all x, y in [b0, b1), z in [c0, c1); either
// (c0, c1) == (b0, b1) or c1 <= b0).  The full block (0, v, 0, v) runs the
// cached plan of all sorted jobs; any other block a list of the sorted jobs
// with at least one such ordering.  Any precision mode (the mixed modes need
// nocc % 8 == 0).
static int run_lno_vjp(const ct_problem *p, int mode, const double *mat, double et_bar, int b0, int b1, int c0,
                       int c1, const ct_grads *g, double *mat_bar, double *e_out, cudaStream_t st) {
    int rc = validate(p, mode);
    if (rc != CT_OK) return rc;
    if (!mat || !mat_bar || !g || !g->mo_energy || !g->t1T || !g->t2T || !g->vooo || !g->fvo || !g->vvop)
        return CT_ERR_NULL;
    const int v = p->nvir;
    if (p->nocc > 64 || b0 < 0 || b1 > v || b0 >= b1 || c0 < 0 || c1 > v || c0 >= c1) return CT_ERR_SHAPE;
    if (!((c0 == b0 && c1 == b1) || c1 <= b0)) return CT_ERR_SHAPE;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    std::lock_guard<std::mutex> lk(Wp->mu);
    return run_lno_vjp_locked(*Wp, p, mode, mat, et_bar, b0, b1, c0, c1, g, mat_bar, e_out, st);
}

// the body of run_lno_vjp, with the workspace lock already held
static int run_lno_vjp_locked(Workspace &W, const ct_problem *p, int mode, const double *mat, double et_bar, int b0,
                              int b1, int c0, int c1, const ct_grads *g, double *mat_bar, double *e_out,
                              cudaStream_t st) {
    int rc = CT_OK;
    const int v = p->nvir;
    const bool full = b0 == 0 && b1 == v && c0 == 0 && c1 == v;
    const int mw = max_wave_jobs(W, p->nocc, mode);
    if ((rc = ensure_common(W, p->nocc, v, mode, mw)) != CT_OK) return rc;
    Plan *P;
    if (full) {
        if (!(P = full_plan(W, p->nocc, v, mw, &rc))) return rc;
    } else {
        auto in = [](int x, int lo, int hi) { return x >= lo && x < hi; };
        std::vector<int> abc;
        for (int a = 0; a < v; ++a)
            for (int b = 0; b <= a; ++b)
                for (int c = 0; c <= b; ++c)
                    if ((in(b, b0, b1) && in(c, c0, c1)) || (in(a, b0, b1) && in(c, c0, c1)) ||
                        (in(a, b0, b1) && in(b, c0, c1))) {
                        abc.push_back(a); abc.push_back(b); abc.push_back(c);
                    }
        W.block.free_dev();
        W.block = Plan();
        for (int &k : W.block_key) k = -1;
        W.block.o = p->nocc; W.block.v = v; W.block.max_wave = mw;
        if (abc.empty()) {
            if (e_out) CT_CK(cudaMemsetAsync(e_out, 0, sizeof(double), st));
            return CT_OK;
        }
        plan_list(W.block, abc.data(), (int)(abc.size() / 3));
        if ((rc = upload_plan(W.block)) != CT_OK) { W.block.free_dev(); W.block = Plan(); return rc; }
        P = &W.block;
    }
    double *part = nullptr;
    CT_CK(cudaMallocAsync(&part, (size_t)mw * p->nocc * p->nocc * sizeof(double), st));
    LnoSel sel;
    sel.mat = mat;
    sel.a0 = 0; sel.a1 = v;
    sel.b0 = b0; sel.b1 = b1; sel.c0 = c0; sel.c1 = c1;
    sel.mat_bar = mat_bar;
    sel.part = part;
    rc = run_plan(W, *P, p, mode, true, et_bar, g, W.job_e, e_out, st, &sel);
    cudaFreeAsync(part, st);
    return rc;
}

static int run_full(const ct_problem *p, int mode, bool vjp, double et_bar, const ct_grads *g,
                    double *e_out, double *job_e_out, cudaStream_t st) {
    return run_sel(p, mode, vjp, et_bar, g, e_out, job_e_out, st, 0, 0, 0, 0, 0);
}


}  // namespace ctb

using namespace ctb;

extern "C" {

int ct_version(void) { return 1; }

const char *ct_status_string(int s) {
    switch (s) {
    case CT_OK: return "ok";
    case CT_ERR_SHAPE: return "shape out of range";
    case CT_ERR_NOMEM: return "out of memory";
    case CT_ERR_CUDA: return "CUDA error";
    case CT_ERR_MODE: return "unknown precision mode";
    case CT_ERR_NULL: return "null pointer";
    case CT_ERR_NO_DEVICE: return "no sm_100 device";
    case CT_ERR_TIMEOUT: return "device wait timed out";
    case CT_ERR_NONFINITE: return "non-finite energy";
    case CT_ERR_SIZE: return "size exceeds a fixed capacity (e.g. the allocation-free scratch array)";
    default: return "unknown status";
    }
}

int ct_energy(const ct_problem *p, int mode, double *e_out, double *job_e_out, void *stream) {
    if (!e_out && !job_e_out) return CT_ERR_NULL;
    return run_full(p, mode, false, 0.0, nullptr, e_out, job_e_out, (cudaStream_t)stream);
}

int ct_energy_vjp(const ct_problem *p, int mode, double et_bar, const ct_grads *g, double *e_out,
                  void *stream) {
    return run_full(p, mode, true, et_bar, g, e_out, nullptr, (cudaStream_t)stream);
}

int ct_energy_block(const ct_problem *p, int mode, int a0, int a1, double *e_out, double *job_e_out,
                    void *stream) {
    if (!e_out && !job_e_out) return CT_ERR_NULL;
    return run_sel(p, mode, false, 0.0, nullptr, e_out, job_e_out, (cudaStream_t)stream, 2, a0, a1, 0, 0);
}

int ct_energy_vjp_block(const ct_problem *p, int mode, double et_bar, const ct_grads *g, int a0, int a1,
                        int b0, int b1, double *e_out, void *stream) {
    return run_sel(p, mode, true, et_bar, g, e_out, nullptr, (cudaStream_t)stream, 1, a0, a1, b0, b1);
}

int ct_energy_jobs(const ct_problem *p, int mode, const int *jobs_abc, int njobs, double *e_out,
                   double *job_e_out, void *stream) {
    if (!e_out && !job_e_out) return CT_ERR_NULL;
    return run_list(p, mode, jobs_abc, njobs, e_out, job_e_out, (cudaStream_t)stream);
}

int ct_lno_energy(const ct_problem *p, const double *mat, int a0, int a1, double *e_out, double *job_e_out,
                  void *stream) {
    return run_lno(p, CT_MODE_FP64, mat, a0, a1, e_out, job_e_out, (cudaStream_t)stream);
}

int ct_t3_init(const ct_problem *p, double *t3_c, double *t3_x, void *stream) {
    int rc = validate(p, CT_MODE_FP64);
    if (rc != CT_OK) return rc;
    if (!t3_c || !t3_x) return CT_ERR_NULL;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    const int mw = max_wave_jobs(W, p->nocc, CT_MODE_FP64);
    if ((rc = ensure_common(W, p->nocc, p->nvir, CT_MODE_FP64, mw)) != CT_OK) return rc;
    Plan *P = full_plan(W, p->nocc, p->nvir, mw, &rc);
    if (!P) return rc;
    return run_plan(W, *P, p, CT_MODE_FP64, false, 0.0, nullptr, W.job_e, nullptr, (cudaStream_t)stream, nullptr,
                    t3_c, t3_x);
}

int ct_lno_energy_mode(const ct_problem *p, int mode, const double *mat, int a0, int a1, double *e_out,
                       double *job_e_out, void *stream) {
    return run_lno(p, mode, mat, a0, a1, e_out, job_e_out, (cudaStream_t)stream);
}

int ct_lno_energy_vjp(const ct_problem *p, const double *mat, double et_bar, const ct_grads *g, double *mat_bar,
                      double *e_out, void *stream) {
    if (!p) return CT_ERR_NULL;
    return run_lno_vjp(p, CT_MODE_FP64, mat, et_bar, 0, p->nvir, 0, p->nvir, g, mat_bar, e_out,
                       (cudaStream_t)stream);
}

int ct_lno_energy_vjp_block(const ct_problem *p, const double *mat, double et_bar, int b0, int b1, int c0, int c1,
                            const ct_grads *g, double *mat_bar, double *e_out, void *stream) {
    return run_lno_vjp(p, CT_MODE_FP64, mat, et_bar, b0, b1, c0, c1, g, mat_bar, e_out, (cudaStream_t)stream);
}

int ct_lno_energy_vjp_mode(const ct_problem *p, int mode, const double *mat, double et_bar, int b0, int b1, int c0,
                           int c1, const ct_grads *g, double *mat_bar, double *e_out, void *stream) {
    return run_lno_vjp(p, mode, mat, et_bar, b0, b1, c0, c1, g, mat_bar, e_out, (cudaStream_t)stream);
}

int ct_profile_enable(int on) {
    Workspace *W = current_ws();
    if (!W) return CT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(W->mu);
    W->prof.clear();
    W->prof.on = on != 0;
    return CT_OK;
}

int ct_profile_read(int kind, double *total_ms, int *launches) {
    if (kind < 0 || kind >= kProfKinds || !total_ms || !launches) return CT_ERR_NULL;
    Workspace *W = current_ws();
    if (!W) return CT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(W->mu);
    double tot = 0.0;
    for (auto &pr : W->prof.ev[kind]) {
        if (cudaEventSynchronize(pr.second) != cudaSuccess) return CT_ERR_CUDA;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.first, pr.second) != cudaSuccess) return CT_ERR_CUDA;
        tot += ms;
    }
    *total_ms = tot;
    *launches = (int)W->prof.ev[kind].size();
    return CT_OK;
}

int ct_profile_reset(void) {
    Workspace *W = current_ws();
    if (!W) return CT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(W->mu);
    W->prof.clear();
    return CT_OK;
}

// releases the workspace of every device this process has used (each with
// that device current), then restores the caller's current device
int ct_release_workspace(void) {
    int cur = -1, ndev = 0;
    if (cudaGetDevice(&cur) != cudaSuccess || cudaGetDeviceCount(&ndev) != cudaSuccess) return CT_OK;
    for (int d = 0; d < ndev && d < kMaxDevices; ++d) {
        Workspace &W = g_ws[d];
        std::lock_guard<std::mutex> lk(W.mu);
        if (W.cc_major < 0) continue;   // never used on this device
        if (cudaSetDevice(d) != cudaSuccess) continue;
        W.release();
        mixed_free_cache();
    }
    if (cur >= 0) cudaSetDevice(cur);
    return CT_OK;
}

long long ct_workspace_bytes(int nocc, int nvir, int mode, int with_vjp) {
    (void)with_vjp;
    if (nocc < 1 || nvir < 1) return CT_ERR_SHAPE;
    long long mw;
    Workspace *W = current_ws();
    if (W) {
        std::lock_guard<std::mutex> lk(W->mu);
        mw = max_wave_jobs(*W, nocc, mode);
    } else {
        Workspace tmp;   // no device: the default budget and SM count
        mw = max_wave_jobs(tmp, nocc, mode);
    }
    return mw * kSlots * (long long)nocc * nocc * nocc * (long long)scratch_elt(mode)
         + (mode == CT_MODE_FP64 ? 0 : (long long)(mw * mixed_extra_bytes_per_job(nocc, mode)))
         + (mode == CT_MODE_FP64 ? 0 : (long long)mixed_operand_bytes(nocc, nvir, mode))
         + n_sorted(nvir) * 8LL + (long long)nocc * nocc * nocc * 4LL;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host-pointer entry points (ctypes path)
// ---------------------------------------------------------------------------
namespace ctb {


struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

static cudaError_t grow(double *&p, size_t &cap, size_t count) {
    if (count <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(1, count) * sizeof(double));
    if (e == cudaSuccess) cap = count;
    else p = nullptr;
    return e;
}

// dst[i] += src[i] on host threads (the += contract of the reference's bars)
static void par_add(double *dst, const double *src, size_t n) {
    const size_t nt = std::max<size_t>(1, std::min<size_t>(32, std::thread::hardware_concurrency()));
    if (n < (1u << 20) || nt == 1) {
        for (size_t i = 0; i < n; ++i) dst[i] += src[i];
        return;
    }
    std::vector<std::thread> th;
    const size_t chunk = (n + nt - 1) / nt;
    for (size_t t = 0; t < nt; ++t) {
        const size_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=] { for (size_t i = b; i < e; ++i) dst[i] += src[i]; });
    }
    for (auto &x : th) x.join();
}

// Device -> host gradient transfers of the host-pointer entries: height rows
// of width doubles (device rows dpitch apart, host rows hpitch apart); the
// host side accumulates (the reference's += contract).
struct Xfer {
    double *host;
    size_t hpitch;
    const double *dev;
    size_t dpitch, width, height;
};

constexpr size_t kStage = size_t(16) << 20;   // doubles per staging half (128 MiB)

// Streams the transfers through the two halves of a pinned staging ring on
// stream st: while the host adds one chunk, the copy of the next one runs.
static int drain_adds(HostPathCache &H, cudaStream_t st, const std::vector<Xfer> &xs) {
    struct Chunk {
        double *host;
        size_t hpitch;
        const double *dev;
        size_t dpitch, width, rows;
    };
    std::vector<Chunk> cs;
    for (const Xfer &x : xs) {
        if (!x.host) return CT_ERR_NULL;
        if (x.width == 0 || x.height == 0) continue;
        if (x.width <= kStage) {
            const size_t per = kStage / x.width;
            for (size_t r = 0; r < x.height; r += per)
                cs.push_back({x.host + r * x.hpitch, x.hpitch, x.dev + r * x.dpitch, x.dpitch, x.width,
                              std::min(per, x.height - r)});
        } else {
            for (size_t r = 0; r < x.height; ++r)
                for (size_t c = 0; c < x.width; c += kStage)
                    cs.push_back({x.host + r * x.hpitch + c, 0, x.dev + r * x.dpitch + c, 0,
                                  std::min(kStage, x.width - c), 1});
        }
    }
    if (cs.empty()) return CT_OK;
    if (H.pin_cap < 2 * kStage) {
        if (H.pin) cudaFreeHost(H.pin);
        H.pin = nullptr;
        H.pin_cap = 0;
        CT_CK(cudaHostAlloc((void **)&H.pin, 2 * kStage * sizeof(double), cudaHostAllocDefault));
        H.pin_cap = 2 * kStage;
    }
    for (auto &e : H.ev)
        if (!e) CT_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    auto enqueue = [&](size_t i) -> int {
        const Chunk &c = cs[i];
        double *buf = H.pin + (i & 1) * kStage;
        if (c.rows == 1)
            CT_CK(cudaMemcpyAsync(buf, c.dev, c.width * 8, cudaMemcpyDeviceToHost, st));
        else
            CT_CK(cudaMemcpy2DAsync(buf, c.width * 8, c.dev, c.dpitch * 8, c.width * 8, c.rows,
                                    cudaMemcpyDeviceToHost, st));
        CT_CK(cudaEventRecord(H.ev[i & 1], st));
        return CT_OK;
    };
    int rc = enqueue(0);
    if (rc == CT_OK && cs.size() > 1) rc = enqueue(1);
    for (size_t i = 0; i < cs.size() && rc == CT_OK; ++i) {
        CT_CK(cudaEventSynchronize(H.ev[i & 1]));
        const Chunk &c = cs[i];
        const double *buf = H.pin + (i & 1) * kStage;
        if (c.rows == 1 || c.hpitch == c.width) {
            par_add(c.host, buf, c.width * c.rows);
        } else {
            for (size_t r = 0; r < c.rows; ++r) par_add(c.host + r * c.hpitch, buf + r * c.width, c.width);
        }
        // this half is free again: the chunk after next may land in it
        if (i + 2 < cs.size()) rc = enqueue(i + 2);
    }
    return rc;
}

static int host_stream(HostPathCache &H, cudaStream_t *st) {
    if (!H.st) CT_CK(cudaStreamCreateWithFlags(&H.st, cudaStreamNonBlocking));
    *st = H.st;
    return CT_OK;
}

static int host_copy_streams(HostPathCache &H) {
    if (!H.st_in) CT_CK(cudaStreamCreateWithFlags(&H.st_in, cudaStreamNonBlocking));
    if (!H.st_out) CT_CK(cudaStreamCreateWithFlags(&H.st_out, cudaStreamNonBlocking));
    return CT_OK;
}

// The reference's slab-block VJP on host arrays (ccsd_t_energy_vjp,
// ccsd_t_vjp.c:332-497, through its 25 arguments), staged so that the host
// copies overlap the device work.  A job (a, b, c) of the block has a in the
// first slab and b in the second; a smallest index c < b0 lies outside both
// slabs and meets the rest of the block only as a job's smallest index.  So
// the jobs run in stages: first those with c >= b0 (they read only the slabs'
// rows of the inputs), then chunks of c < b0 of about one wave each, whose
// inputs are the vvop rows and columns on c and the t2T / vooo rows c, and
// whose gradients (the same rows and columns) are final once the chunk's
// waves are done.  The copies in run one stage ahead on their own stream; a
// finished chunk's gradients come back through the pinned ring and are added
// on the host while the next chunk computes; the slabs' rows and the small
// arrays come back at the end.  CTB_HOST_TIMING=1 prints the phase times to
// stderr.
static int host_block_vjp(double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                          double et_bar, int nocc, int nvir, int a0, int a1, int b0, int b1,
                          void *cache_row_a, void *cache_col_a, void *cache_row_b, void *cache_col_b,
                          double *mo_energy_bar, double *t1T_bar, double *t2T_bar, double *vooo_bar,
                          double *fvo_bar, double *cache_row_a_bar, double *cache_col_a_bar,
                          double *cache_row_b_bar, double *cache_col_b_bar, int mode) {
    if (!mo_energy || !t1T || !t2T || !vooo || !fvo || !cache_row_a) return CT_ERR_NULL;
    if (nocc < 1 || nocc > 255 || nvir < 1 || nvir > 1024) return CT_ERR_SHAPE;
    if (a0 < 0 || a1 > nvir || a0 >= a1 || b0 < 0 || b1 > a1 || b0 >= b1) return CT_ERR_SHAPE;
    if (!(b1 <= a0 || (b0 == a0 && b1 == a1))) return CT_ERR_SHAPE;
    if (mode != CT_MODE_FP64 && mode != CT_MODE_TF32 && mode != CT_MODE_BF16X3) return CT_ERR_MODE;
    int rc = CT_OK;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    const long long o = nocc, v = nvir, n = o + v, onb = o * n, zrow = v * o * o, xrow = o * o * o;
    const size_t sz_mo = n, sz_t1 = v * o, sz_t2 = v * v * o * o, sz_vooo = v * o * o * o, sz_vvop = v * v * onb;
    const size_t sizes[HostPathCache::NBUF] = {sz_mo, sz_t1, sz_t2, sz_vooo, sz_t1, sz_vvop};
    // the block's caches: rows x in [x0, x1), columns y in [y0, y1) of vvop,
    // each (x, y) entry o*n doubles; only these are read by the block's jobs
    // and written in its vvop gradient
    struct Region { void *h; double *hbar; int x0, x1, y0, y1; };
    std::vector<Region> regs;
    const bool use_col_a = a0 > 0, use_row_b = b1 <= a0, use_col_b = use_row_b && b0 > 0;
    regs.push_back({cache_row_a, cache_row_a_bar, a0, a1, 0, a1});
    if (use_col_a) regs.push_back({cache_col_a, cache_col_a_bar, 0, a0, a0, a1});
    if (use_row_b) regs.push_back({cache_row_b, cache_row_b_bar, b0, b1, 0, b1});
    if (use_col_b) regs.push_back({cache_col_b, cache_col_b_bar, 0, b0, b0, b1});
    for (auto &r : regs)
        if (!r.h || !r.hbar) return CT_ERR_NULL;
    if (!mo_energy_bar || !t1T_bar || !t2T_bar || !vooo_bar || !fvo_bar) return CT_ERR_NULL;
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    HostPathCache &H = W.hp;
    const bool timing = std::getenv("CTB_HOST_TIMING") != nullptr;
    const auto t_start = std::chrono::steady_clock::now();
    for (int i = 0; i < HostPathCache::NBUF; ++i) {
        CT_CK(grow(H.in[i], H.in_cap[i], sizes[i]));
        CT_CK(grow(H.bar[i], H.bar_cap[i], sizes[i]));
    }
    cudaStream_t st = nullptr;
    if ((rc = host_stream(H, &st)) != CT_OK) return rc;
    if ((rc = host_copy_streams(H)) != CT_OK) return rc;
    double **din = H.in, **dbar = H.bar;
    const int mw = max_wave_jobs(W, nocc, mode);
    if ((rc = ensure_common(W, nocc, nvir, mode, mw)) != CT_OK) return rc;

    // stages: 0 = the jobs with c >= b0 (rows [b0, a1) of the inputs); k >= 1 =
    // the chunk c in [(k-1) cw, min(k cw, b0)), about one wave of jobs
    const int cf = b0;
    std::vector<std::vector<int>> sjobs;
    int cw = 1;
    const int S = block_stages(a0, a1, b0, b1, mw, &cw, sjobs);
    auto rows = [&](int s, int &r0, int &r1) {
        if (s == 0) { r0 = cf; r1 = a1; }
        else { r0 = (s - 1) * cw; r1 = std::min(cf, s * cw); }
    };
    // the part of a cache a stage covers: row caches (y from 0) by columns,
    // column caches by rows
    auto part = [&](const Region &r, int s, int &x0, int &x1, int &y0, int &y1) {
        int r0, r1;
        rows(s, r0, r1);
        x0 = r.x0; x1 = r.x1; y0 = r.y0; y1 = r.y1;
        if (r.y0 == 0) { y0 = std::max(r.y0, r0); y1 = std::min(r.y1, r1); }
        else { x0 = std::max(r.x0, r0); x1 = std::min(r.x1, r1); }
        return x1 > x0 && y1 > y0;
    };
    std::vector<Plan> plans(S);
    std::vector<cudaEvent_t> in_ev(S, nullptr), done_ev(S, nullptr);
    cudaEvent_t t_ev[2] = {nullptr, nullptr};
    MixedOperands mo{};
    bool mixed_set = false;
    // every exit: the streams drained before the plans' tables and the events go
    auto finish = [&](int code) {
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(H.st_in);
        cudaStreamSynchronize(H.st_out);
        if (mixed_set) mixed_release(&mo, st);
        for (auto &P : plans) P.free_dev();
        for (auto &e : in_ev) if (e) cudaEventDestroy(e);
        for (auto &e : done_ev) if (e) cudaEventDestroy(e);
        for (auto &e : t_ev) if (e) cudaEventDestroy(e);
        return code;
    };
    for (int k = 0; k < S; ++k) {
        plans[k].o = nocc; plans[k].v = nvir; plans[k].max_wave = mw;
        if (!sjobs[k].empty()) {
            plan_grouped(plans[k], sjobs[k]);
            if ((rc = upload_plan(plans[k])) != CT_OK) return finish(rc);
        }
        if (cudaEventCreateWithFlags(&in_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&done_ev[k], cudaEventDisableTiming) != cudaSuccess)
            return finish(CT_ERR_CUDA);
    }
    if (timing)
        for (auto &e : t_ev)
            if (cudaEventCreate(&e) != cudaSuccess) return finish(CT_ERR_CUDA);
#define HB_CK(x) do { if ((x) != cudaSuccess) return finish(CT_ERR_CUDA); } while (0)
    // gradients start at zero (device side only: rows [0, a1) and the caches)
    double *hbar_small[3] = {mo_energy_bar, t1T_bar, fvo_bar};
    const int small_idx[3] = {HostPathCache::MO, HostPathCache::T1, HostPathCache::FVO};
    for (int i : small_idx) HB_CK(cudaMemsetAsync(dbar[i], 0, sizes[i] * 8, st));
    HB_CK(cudaMemsetAsync(dbar[HostPathCache::T2], 0, a1 * zrow * 8, st));
    HB_CK(cudaMemsetAsync(dbar[HostPathCache::VOOO], 0, a1 * xrow * 8, st));
    for (auto &r : regs)
        HB_CK(cudaMemset2DAsync(dbar[HostPathCache::VVOP] + ((size_t)r.x0 * v + r.y0) * onb, (size_t)v * onb * 8, 0,
                                (size_t)(r.y1 - r.y0) * onb * 8, r.x1 - r.x0, st));
    HB_CK(cudaMemsetAsync(W.job_e, 0, n_sorted(v) * sizeof(double), st));
    if (timing) HB_CK(cudaEventRecord(t_ev[0], st));
    const double *hin_small[3] = {mo_energy, t1T, fvo};
    auto copy_in = [&](int s) -> int {
        cudaStream_t cs = H.st_in;
        int r0, r1;
        rows(s, r0, r1);
        if (s == 0)
            for (int k = 0; k < 3; ++k)
                CT_CK(cudaMemcpyAsync(din[small_idx[k]], hin_small[k], sizes[small_idx[k]] * 8,
                                      cudaMemcpyHostToDevice, cs));
        if (r1 > r0) {
            CT_CK(cudaMemcpyAsync(din[HostPathCache::T2] + r0 * zrow, t2T + r0 * zrow, (r1 - r0) * zrow * 8,
                                  cudaMemcpyHostToDevice, cs));
            CT_CK(cudaMemcpyAsync(din[HostPathCache::VOOO] + r0 * xrow, vooo + r0 * xrow, (r1 - r0) * xrow * 8,
                                  cudaMemcpyHostToDevice, cs));
        }
        for (auto &r : regs) {
            int x0, x1, y0, y1;
            if (!part(r, s, x0, x1, y0, y1)) continue;
            const size_t hp = (size_t)(r.y1 - r.y0) * onb;
            const double *h = static_cast<const double *>(r.h) + ((size_t)(x0 - r.x0) * (r.y1 - r.y0) + (y0 - r.y0)) * onb;
            CT_CK(cudaMemcpy2DAsync(din[HostPathCache::VVOP] + ((size_t)x0 * v + y0) * onb, (size_t)v * onb * 8, h,
                                    hp * 8, (size_t)(y1 - y0) * onb * 8, x1 - x0, cudaMemcpyHostToDevice, cs));
        }
        CT_CK(cudaEventRecord(in_ev[s], cs));
        return CT_OK;
    };
    // stage s's gradients, once its waves are done, added into the caller's arrays
    auto drain = [&](int s) -> int {
        std::vector<Xfer> xs;
        int r0, r1;
        rows(s, r0, r1);
        if (s == 0)
            for (int k = 0; k < 3; ++k)
                xs.push_back({hbar_small[k], sizes[small_idx[k]], dbar[small_idx[k]], sizes[small_idx[k]],
                              sizes[small_idx[k]], 1});
        if (r1 > r0) {
            const size_t nz = (size_t)(r1 - r0) * zrow, nx = (size_t)(r1 - r0) * xrow;
            xs.push_back({t2T_bar + r0 * zrow, nz, dbar[HostPathCache::T2] + r0 * zrow, nz, nz, 1});
            xs.push_back({vooo_bar + r0 * xrow, nx, dbar[HostPathCache::VOOO] + r0 * xrow, nx, nx, 1});
        }
        for (auto &r : regs) {
            int x0, x1, y0, y1;
            if (!part(r, s, x0, x1, y0, y1)) continue;
            const size_t hp = (size_t)(r.y1 - r.y0) * onb;
            xs.push_back({r.hbar + ((size_t)(x0 - r.x0) * (r.y1 - r.y0) + (y0 - r.y0)) * onb, hp,
                          dbar[HostPathCache::VVOP] + ((size_t)x0 * v + y0) * onb, (size_t)v * onb,
                          (size_t)(y1 - y0) * onb, (size_t)(x1 - x0)});
        }
        CT_CK(cudaStreamWaitEvent(H.st_out, done_ev[s == 0 ? S - 1 : s], 0));
        return drain_adds(H, H.st_out, xs);
    };
    ct_problem prob{nocc, nvir, din[HostPathCache::MO], din[HostPathCache::T1], din[HostPathCache::T2],
                    din[HostPathCache::VOOO], din[HostPathCache::FVO], din[HostPathCache::VVOP]};
    ct_grads gr{dbar[HostPathCache::MO], dbar[HostPathCache::T1], dbar[HostPathCache::T2],
                dbar[HostPathCache::VOOO], dbar[HostPathCache::FVO], dbar[HostPathCache::VVOP]};
    const EpiArgs ea = epi_args(W, &prob, true, et_bar, &gr, W.job_e, nullptr);
    if (mode != CT_MODE_FP64) {
        if ((rc = mixed_setup(&prob, mode, &mo, st)) != CT_OK) return finish(rc);
        mixed_set = true;
    }
    if ((rc = copy_in(0)) != CT_OK) return finish(rc);
    for (int s = 0; s < S; ++s) {
        HB_CK(cudaStreamWaitEvent(st, in_ev[s], 0));
        if (mixed_set) {
            MixedRegion mr;
            rows(s, mr.z0, mr.z1);
            mr.x0 = mr.z0; mr.x1 = mr.z1;
            for (auto &r : regs) {
                int x0, x1, y0, y1;
                if (!part(r, s, x0, x1, y0, y1)) continue;
                int *q = mr.rect[mr.nrect++];
                q[0] = x0; q[1] = x1; q[2] = y0; q[3] = y1;
            }
            if ((rc = mixed_convert(&prob, mo, mr, st)) != CT_OK) return finish(rc);
        }
        if (plans[s].d_jobs && (rc = run_waves(W, plans[s], &prob, mode, true, &gr, ea, mo, nullptr, st)) != CT_OK)
            return finish(rc);
        HB_CK(cudaEventRecord(done_ev[s], st));
        if (s + 1 < S && (rc = copy_in(s + 1)) != CT_OK) return finish(rc);
        if (s >= 2 && (rc = drain(s - 1)) != CT_OK) return finish(rc);   // chunk s-1 is final
    }
    if (timing) HB_CK(cudaEventRecord(t_ev[1], st));
    if (S >= 2 && (rc = drain(S - 1)) != CT_OK) return finish(rc);
    if ((rc = drain(0)) != CT_OK) return finish(rc);
    if (mixed_set) {
        if ((rc = mixed_check_error(st)) != CT_OK) return finish(rc);
    }
    if (timing) {
        cudaStreamSynchronize(st);
        float dev = 0.f;
        cudaEventElapsedTime(&dev, t_ev[0], t_ev[1]);
        std::fprintf(stderr, "ctb host path: total %.1f ms (wall); %d stages; device span (first copy wait to "
                     "last wave) %.1f ms\n",
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count(),
                     S, dev);
    }
#undef HB_CK
    return finish(CT_OK);
}

// Host-pointer LNO backward block (lnoccsdt_energy_vjp, lno_ccsd_t_vjp.c:400-566)
// on the caches pyscfad's driver cuts (pyscfad/lno/ccsd_t.py:194-220): for
// each slab [s0, s1) the row cache vvop[s0:s1, :] and the column cache
// vvop[:, s0:s1] (the same array when the slab is [0, nvir)).  They are
// placed into a device vvop; the vvop gradient comes back so that each
// (x, y) pair is added to exactly one of the cache gradients (rows of the
// first slab, then its columns, then the second slab's rows and columns),
// which is what the driver's sums over the caches need.
static int host_lno_block_vjp(double *mat, double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                              double et_bar, int nocc, int nvir, int b0, int b1, int c0, int c1,
                              void *cache_row_a, void *cache_col_a, void *cache_row_b, void *cache_col_b,
                              double *mat_bar, double *mo_energy_bar, double *t1T_bar, double *t2T_bar,
                              double *vooo_bar, double *fvo_bar, double *cache_row_a_bar, double *cache_col_a_bar,
                              double *cache_row_b_bar, double *cache_col_b_bar) {
    if (!mat || !mo_energy || !t1T || !t2T || !vooo || !fvo || !mat_bar || !mo_energy_bar || !t1T_bar ||
        !t2T_bar || !vooo_bar || !fvo_bar)
        return CT_ERR_NULL;
    if (nocc < 1 || nocc > 64 || nvir < 1 || nvir > 1024) return CT_ERR_SHAPE;
    if (b0 < 0 || b1 > nvir || b0 >= b1 || c0 < 0 || c1 > nvir || c0 >= c1) return CT_ERR_SHAPE;
    if (!((c0 == b0 && c1 == b1) || c1 <= b0)) return CT_ERR_SHAPE;
    int rc = CT_OK;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    struct Slab { int s0, s1; const double *row, *col; double *row_bar, *col_bar; };
    std::vector<Slab> slabs;
    slabs.push_back({b0, b1, (const double *)cache_row_a, (const double *)cache_col_a, cache_row_a_bar,
                     cache_col_a_bar});
    if (!(c0 == b0 && c1 == b1))
        slabs.push_back({c0, c1, (const double *)cache_row_b, (const double *)cache_col_b, cache_row_b_bar,
                         cache_col_b_bar});
    for (auto &sl : slabs) {
        const bool fullslab = sl.s0 == 0 && sl.s1 == nvir;
        if (!sl.row || !sl.row_bar || (!fullslab && (!sl.col || !sl.col_bar))) return CT_ERR_NULL;
    }
    const long long o = nocc, v = nvir, n = o + v, onb = o * n;
    const size_t sz_mo = n, sz_t1 = v * o, sz_t2 = v * v * o * o, sz_vooo = v * o * o * o, sz_vvop = v * v * onb;
    const size_t sizes[HostPathCache::NBUF] = {sz_mo, sz_t1, sz_t2, sz_vooo, sz_t1, sz_vvop};
    Workspace &W = *Wp;
    std::lock_guard<std::mutex> lk(W.mu);
    HostPathCache &H = W.hp;
    for (int i = 0; i < HostPathCache::NBUF; ++i) {
        CT_CK(grow(H.in[i], H.in_cap[i], sizes[i]));
        CT_CK(grow(H.bar[i], H.bar_cap[i], sizes[i]));
    }
    double **din = H.in, **dbar = H.bar;
    CT_CK(cudaMemcpy(din[HostPathCache::MO], mo_energy, sz_mo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(din[HostPathCache::T1], t1T, sz_t1 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(din[HostPathCache::T2], t2T, sz_t2 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(din[HostPathCache::VOOO], vooo, sz_vooo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(din[HostPathCache::FVO], fvo, sz_t1 * 8, cudaMemcpyHostToDevice));
    for (int i = 0; i < HostPathCache::NBUF; ++i)
        if (i != HostPathCache::VVOP) CT_CK(cudaMemset(dbar[i], 0, sizes[i] * 8));
    double *dvv = din[HostPathCache::VVOP], *dvb = dbar[HostPathCache::VVOP];
    for (auto &sl : slabs) {
        const long long ds = sl.s1 - sl.s0;
        CT_CK(cudaMemcpy(dvv + sl.s0 * v * onb, sl.row, (size_t)(ds * v * onb) * 8, cudaMemcpyHostToDevice));
        CT_CK(cudaMemset(dvb + sl.s0 * v * onb, 0, (size_t)(ds * v * onb) * 8));
        if (!(sl.s0 == 0 && sl.s1 == nvir)) {
            CT_CK(cudaMemcpy2D(dvv + sl.s0 * onb, (size_t)(v * onb) * 8, sl.col, (size_t)(ds * onb) * 8,
                               (size_t)(ds * onb) * 8, (size_t)v, cudaMemcpyHostToDevice));
            CT_CK(cudaMemset2D(dvb + sl.s0 * onb, (size_t)(v * onb) * 8, 0, (size_t)(ds * onb) * 8, (size_t)v));
        }
    }
    DevBuf dmat, dmb;
    CT_CK(cudaMalloc(&dmat.p, o * o * 8));
    CT_CK(cudaMalloc(&dmb.p, o * o * 8));
    CT_CK(cudaMemcpy(dmat.p, mat, o * o * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemset(dmb.p, 0, o * o * 8));
    ct_problem prob{nocc, nvir, din[HostPathCache::MO], din[HostPathCache::T1], din[HostPathCache::T2],
                    din[HostPathCache::VOOO], din[HostPathCache::FVO], dvv};
    ct_grads gr{dbar[HostPathCache::MO], dbar[HostPathCache::T1], dbar[HostPathCache::T2],
                dbar[HostPathCache::VOOO], dbar[HostPathCache::FVO], dvb};
    if ((rc = run_lno_vjp_locked(W, &prob, CT_MODE_FP64, (const double *)dmat.p, et_bar, b0, b1, c0, c1, &gr, (double *)dmb.p,
                                 nullptr, 0)) != CT_OK)
        return rc;
    if (cudaDeviceSynchronize() != cudaSuccess) return CT_ERR_CUDA;
    // device -> pinned -> += host, a height x width block (elements) at the given pitches
    auto add_2d = [&](double *host, size_t hpitch, const double *dev, size_t dpitch, size_t width,
                      size_t height) -> int {
        if (width == 0 || height == 0) return CT_OK;
        const size_t need = width * height;
        if (need > H.pin_cap) {
            if (H.pin) cudaFreeHost(H.pin);
            H.pin = nullptr;
            H.pin_cap = 0;
            CT_CK(cudaHostAlloc((void **)&H.pin, need * 8, cudaHostAllocDefault));
            H.pin_cap = need;
        }
        CT_CK(cudaMemcpy2D(H.pin, width * 8, dev, dpitch * 8, width * 8, height, cudaMemcpyDeviceToHost));
        if (hpitch == width) {
            par_add(host, H.pin, need);
        } else {
            for (size_t r = 0; r < height; ++r) par_add(host + r * hpitch, H.pin + r * width, width);
        }
        return CT_OK;
    };
    if ((rc = add_2d(mo_energy_bar, sz_mo, dbar[HostPathCache::MO], sz_mo, sz_mo, 1)) != CT_OK) return rc;
    if ((rc = add_2d(t1T_bar, sz_t1, dbar[HostPathCache::T1], sz_t1, sz_t1, 1)) != CT_OK) return rc;
    if ((rc = add_2d(t2T_bar, sz_t2, dbar[HostPathCache::T2], sz_t2, sz_t2, 1)) != CT_OK) return rc;
    if ((rc = add_2d(vooo_bar, sz_vooo, dbar[HostPathCache::VOOO], sz_vooo, sz_vooo, 1)) != CT_OK) return rc;
    if ((rc = add_2d(fvo_bar, sz_t1, dbar[HostPathCache::FVO], sz_t1, sz_t1, 1)) != CT_OK) return rc;
    if ((rc = add_2d(mat_bar, o * o, (const double *)dmb.p, o * o, o * o, 1)) != CT_OK) return rc;
    // vvop gradient: each pair to one cache gradient.  Pairs claimed so far:
    // rows of earlier slabs (all y) and columns of earlier slabs (other x).
    std::vector<std::pair<long long, long long>> rows_claimed, cols_claimed;
    auto minus = [](long long lo, long long hi, const std::vector<std::pair<long long, long long>> &cut) {
        std::vector<std::pair<long long, long long>> out{{lo, hi}};
        for (auto &c : cut) {
            std::vector<std::pair<long long, long long>> nx;
            for (auto &iv : out) {
                if (c.second <= iv.first || c.first >= iv.second) { nx.push_back(iv); continue; }
                if (iv.first < c.first) nx.push_back({iv.first, c.first});
                if (c.second < iv.second) nx.push_back({c.second, iv.second});
            }
            out.swap(nx);
        }
        return out;
    };
    for (auto &sl : slabs) {
        const long long ds = sl.s1 - sl.s0;
        // rows [s0, s1), y outside the columns claimed by earlier slabs
        for (auto &yi : minus(0, v, cols_claimed))
            if ((rc = add_2d(sl.row_bar + yi.first * onb, (size_t)(v * onb), dvb + (sl.s0 * v + yi.first) * onb,
                             (size_t)(v * onb), (size_t)((yi.second - yi.first) * onb), (size_t)ds)) != CT_OK)
                return rc;
        rows_claimed.push_back({sl.s0, sl.s1});
        if (!(sl.s0 == 0 && sl.s1 == nvir)) {
            // columns [s0, s1), x outside every claimed row range
            for (auto &xi : minus(0, v, rows_claimed))
                if ((rc = add_2d(sl.col_bar + xi.first * ds * onb, (size_t)(ds * onb),
                                 dvb + (xi.first * v + sl.s0) * onb, (size_t)(v * onb), (size_t)(ds * onb),
                                 (size_t)(xi.second - xi.first))) != CT_OK)
                    return rc;
        }
        cols_claimed.push_back({sl.s0, sl.s1});
    }
    return CT_OK;
}

}  // namespace ctb

extern "C" {

int ctb_ccsd_t_energy_vjp(double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                          double et_bar, int nocc, int nvir, int a0, int a1, int b0, int b1,
                          void *cache_row_a, void *cache_col_a, void *cache_row_b, void *cache_col_b,
                          double *mo_energy_bar, double *t1T_bar, double *t2T_bar, double *vooo_bar,
                          double *fvo_bar, double *cache_row_a_bar, double *cache_col_a_bar,
                          double *cache_row_b_bar, double *cache_col_b_bar) {
    return host_block_vjp(mo_energy, t1T, t2T, vooo, fvo, et_bar, nocc, nvir, a0, a1, b0, b1, cache_row_a,
                          cache_col_a, cache_row_b, cache_col_b, mo_energy_bar, t1T_bar, t2T_bar, vooo_bar,
                          fvo_bar, cache_row_a_bar, cache_col_a_bar, cache_row_b_bar, cache_col_b_bar,
                          CT_MODE_FP64);
}

int ctb_ccsd_t_energy_vjp_mode(double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                               double et_bar, int nocc, int nvir, int a0, int a1, int b0, int b1,
                               void *cache_row_a, void *cache_col_a, void *cache_row_b, void *cache_col_b,
                               double *mo_energy_bar, double *t1T_bar, double *t2T_bar, double *vooo_bar,
                               double *fvo_bar, double *cache_row_a_bar, double *cache_col_a_bar,
                               double *cache_row_b_bar, double *cache_col_b_bar, int mode) {
    if (mode != CT_MODE_FP64 && mode != CT_MODE_TF32 && mode != CT_MODE_BF16X3) return CT_ERR_MODE;
    return host_block_vjp(mo_energy, t1T, t2T, vooo, fvo, et_bar, nocc, nvir, a0, a1, b0, b1, cache_row_a,
                          cache_col_a, cache_row_b, cache_col_b, mo_energy_bar, t1T_bar, t2T_bar, vooo_bar,
                          fvo_bar, cache_row_a_bar, cache_col_a_bar, cache_row_b_bar, cache_col_b_bar, mode);
}

int ctb_ccsd_t_energy(double *e_tot, double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                      int nocc, int nvir, int a0, int a1, double *vvop, int mode) {
    using namespace ctb;
    if (!e_tot || !mo_energy || !t1T || !t2T || !vooo || !fvo || !vvop) return CT_ERR_NULL;
    if (nocc < 1 || nocc > 255 || nvir < 1 || nvir > 1024 || a0 < 0 || a1 > nvir || a0 >= a1)
        return CT_ERR_SHAPE;
    if (mode != CT_MODE_FP64 && mode != CT_MODE_TF32 && mode != CT_MODE_BF16X3) return CT_ERR_MODE;
    int rc = CT_OK;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    const long long o = nocc, v = nvir, n = o + v;
    const size_t sz_mo = n, sz_t1 = v * o, sz_t2 = v * v * o * o, sz_vooo = v * o * o * o, sz_vvop = v * v * o * n;
    DevBuf dmo, dt1, dt2, dvooo, dfvo, dvvop;
    CT_CK(cudaMalloc(&dmo.p, sz_mo * 8));
    CT_CK(cudaMalloc(&dt1.p, sz_t1 * 8));
    CT_CK(cudaMalloc(&dt2.p, sz_t2 * 8));
    CT_CK(cudaMalloc(&dvooo.p, sz_vooo * 8));
    CT_CK(cudaMalloc(&dfvo.p, sz_t1 * 8));
    CT_CK(cudaMalloc(&dvvop.p, sz_vvop * 8));
    CT_CK(cudaMemcpy(dmo.p, mo_energy, sz_mo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dt1.p, t1T, sz_t1 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dt2.p, t2T, sz_t2 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dvooo.p, vooo, sz_vooo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dfvo.p, fvo, sz_t1 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dvvop.p, vvop, sz_vvop * 8, cudaMemcpyHostToDevice));
    ct_problem prob{nocc, nvir, (double *)dmo.p, (double *)dt1.p, (double *)dt2.p, (double *)dvooo.p,
                    (double *)dfvo.p, (double *)dvvop.p};
    double e = 0.0;
    {
        Workspace &W = *Wp;
        std::lock_guard<std::mutex> lk(W.mu);
        const int mw = max_wave_jobs(W, nocc, mode);
        if ((rc = ensure_common(W, nocc, nvir, mode, mw)) != CT_OK) return rc;
        Plan P;
        P.o = nocc; P.v = nvir; P.max_wave = mw;
        plan_aslab(P, a0, a1);
        if ((rc = upload_plan(P)) != CT_OK) { P.free_dev(); return rc; }
        rc = run_plan(W, P, &prob, mode, false, 0.0, nullptr, W.job_e, W.e_tmp, 0);
        cudaError_t se = cudaDeviceSynchronize();
        P.free_dev();
        if (rc != CT_OK) return rc;
        if (se != cudaSuccess) return CT_ERR_CUDA;
        CT_CK(cudaMemcpy(&e, W.e_tmp, sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (!std::isfinite(e)) return CT_ERR_NONFINITE;
    *e_tot += e;
    return CT_OK;
}

int ctb_lnoccsdt_energy_vjp(double *mat, double *mo_energy, double *t1T, double *t2T, double *vooo, double *fvo,
                            double et_bar, int nocc, int nvir, int b0, int b1, int c0, int c1, void *cache_row_a,
                            void *cache_col_a, void *cache_row_b, void *cache_col_b, double *mat_bar,
                            double *mo_energy_bar, double *t1T_bar, double *t2T_bar, double *vooo_bar,
                            double *fvo_bar, double *cache_row_a_bar, double *cache_col_a_bar,
                            double *cache_row_b_bar, double *cache_col_b_bar) {
    return host_lno_block_vjp(mat, mo_energy, t1T, t2T, vooo, fvo, et_bar, nocc, nvir, b0, b1, c0, c1, cache_row_a,
                              cache_col_a, cache_row_b, cache_col_b, mat_bar, mo_energy_bar, t1T_bar, t2T_bar,
                              vooo_bar, fvo_bar, cache_row_a_bar, cache_col_a_bar, cache_row_b_bar,
                              cache_col_b_bar);
}

int ctb_lnoccsdt_contract(double *e_tot, double *mat, double *mo_energy, double *t1T, double *t2T, double *vooo,
                          double *fvo, int nocc, int nvir, int a0, int a1, double *vvop) {
    using namespace ctb;
    if (!e_tot || !mat || !mo_energy || !t1T || !t2T || !vooo || !fvo || !vvop) return CT_ERR_NULL;
    if (nocc < 1 || nocc > 64 || nvir < 1 || nvir > 1024 || a0 < 0 || a1 > nvir || a0 >= a1) return CT_ERR_SHAPE;
    int rc = CT_OK;
    Workspace *Wp = device_ws(&rc);
    if (!Wp) return rc;
    const long long o = nocc, v = nvir, n = o + v;
    const size_t sz_mo = n, sz_t1 = v * o, sz_t2 = v * v * o * o, sz_vooo = v * o * o * o, sz_vvop = v * v * o * n;
    DevBuf dmo, dt1, dt2, dvooo, dfvo, dvvop, dmat, de;
    CT_CK(cudaMalloc(&dmo.p, sz_mo * 8));
    CT_CK(cudaMalloc(&dt1.p, sz_t1 * 8));
    CT_CK(cudaMalloc(&dt2.p, sz_t2 * 8));
    CT_CK(cudaMalloc(&dvooo.p, sz_vooo * 8));
    CT_CK(cudaMalloc(&dfvo.p, sz_t1 * 8));
    CT_CK(cudaMalloc(&dvvop.p, sz_vvop * 8));
    CT_CK(cudaMalloc(&dmat.p, o * o * 8));
    CT_CK(cudaMalloc(&de.p, 8));
    CT_CK(cudaMemcpy(dmo.p, mo_energy, sz_mo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dt1.p, t1T, sz_t1 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dt2.p, t2T, sz_t2 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dvooo.p, vooo, sz_vooo * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dfvo.p, fvo, sz_t1 * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dvvop.p, vvop, sz_vvop * 8, cudaMemcpyHostToDevice));
    CT_CK(cudaMemcpy(dmat.p, mat, o * o * 8, cudaMemcpyHostToDevice));
    ct_problem prob{nocc, nvir, (double *)dmo.p, (double *)dt1.p, (double *)dt2.p, (double *)dvooo.p,
                    (double *)dfvo.p, (double *)dvvop.p};
    if ((rc = run_lno(&prob, CT_MODE_FP64, (const double *)dmat.p, a0, a1, (double *)de.p, nullptr, 0)) != CT_OK)
        return rc;
    double e = 0.0;
    CT_CK(cudaMemcpy(&e, de.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (!std::isfinite(e)) return CT_ERR_NONFINITE;
    *e_tot += e;
    return CT_OK;
}

}  // extern "C"
