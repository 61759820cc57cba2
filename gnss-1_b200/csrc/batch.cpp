// batch.cpp -- ensembles and the serving loop, built on the C ABI of
// gnss_b200.h.
//
// Ensemble: many independent jets (uneven grids, Reynolds and Schmidt numbers)
// stepped together.  Members of one geometry (grid, precision, scalars,
// scheme, drift coefficient) form groups of up to GNSS_BATCH_MAX whose state,
// history and scratch lie at fixed strides in one buffer per group.  A group
// steps either member by member (each member a unit of its own) or, where
// its kernels allow, as one batched launch per stage (gnss_step_batch: the
// group is one unit); the autotuner picks per group.  Units are spread over a
// few non-blocking streams; the steps of all units are captured once into one
// CUDA graph (one branch per stream) and replayed, so a block of steps of the
// whole ensemble is one launch.
//
// Server: continuous batching.  Submitted requests wait in arrival order; a
// scheduler thread admits them as soon as an active slot and enough of the
// device-memory budget are free, and advances every active request on its own
// stream in chunks of steps (one graph launch per chunk).  Device memory of a
// request (state, history, scratch) is stream-ordered (cudaMallocAsync /
// cudaFreeAsync), so admissions and completions never synchronise the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "gnss_b200.h"
#include "internal.h"

namespace {

size_t elem_bytes(const gnss_config &c) { return c.precision == GNSS_FP64 ? 16 : 8; }
size_t field_bytes_of(const gnss_config &c) {
    return (size_t)c.nx * c.ny * (c.nz / 2 + 1) * elem_bytes(c);
}
int nfields_of(const gnss_config &c) { return 3 + c.n_scalars; }
size_t round256(size_t b) { return (b + 255) / 256 * 256; }

gnss_fields fields_at(void *base, size_t fb, int nf) {
    void *p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < nf; ++q) p[q] = static_cast<char *>(base) + (size_t)q * fb;
    return gnss_fields{p[0], p[1], p[2], p[3], p[4]};
}

struct Member {
    gnss_config cfg{};
    gnss_ctx *ctx = nullptr;
    void *buf = nullptr;   // state (nf fields) then history (nf fields), in its group's buffer
    gnss_fields state{}, hist{};
    int group = 0;
    int branch = 0;        // stream of the member's own steps
};

// Members of one geometry stepped by one batched launch per stage (or, for a
// scheme the batches do not serve, one after another).
struct Group {
    std::vector<int> members;
    void *buf = nullptr;       // the members' state and history slots
    void *scratch = nullptr;   // the members' scratch slices
    size_t slot = 0;           // bytes per member slot (state + history), a multiple of 256
    size_t slice = 0;          // bytes per member scratch slice, a multiple of 256
    bool batched = false;      // one batched launch per stage (else the members' own steps)
    int branch = 0;            // stream of the batched steps
    double points = 0.0;
    long long launches_per_step = 0;
};

bool same_geometry(const gnss_config &a, const gnss_config &b) {
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.precision == b.precision &&
           a.n_scalars == b.n_scalars && a.scheme == b.scheme && a.alpha == b.alpha && a.lx == b.lx &&
           a.ly == b.ly && a.lz == b.lz && a.alias_filter == b.alias_filter;
}

}  // namespace

// ====================================================================== ensemble
struct gnss_ensemble {
    int device = 0;
    std::vector<Member> m;
    std::vector<Group> groups;
    int nbranch = 1;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> ev_join;
    cudaEvent_t ev_fork = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int g_steps = 0;
    long long steps_done = 0;
};

static void ensemble_free(gnss_ensemble *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaDeviceSynchronize();
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    for (Member &mb : e->m)
        if (mb.ctx) gnss_destroy(mb.ctx);
    for (Group &g : e->groups) {
        if (g.buf) cudaFree(g.buf);
        if (g.scratch) cudaFree(g.scratch);
    }
    for (cudaStream_t s : e->streams) if (s) cudaStreamDestroy(s);
    for (cudaEvent_t ev : e->ev_join) if (ev) cudaEventDestroy(ev);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->cap) cudaStreamDestroy(e->cap);
    delete e;
}

// Units (a batched group, or a member stepping on its own) to branches: longest
// processing time first, each unit (by points) to the least-loaded branch.
static void assign_branches(gnss_ensemble *e) {
    struct Unit { double pts; int group; int member; };
    std::vector<Unit> units;
    for (size_t gi = 0; gi < e->groups.size(); ++gi) {
        const Group &g = e->groups[gi];
        if (g.batched) {
            units.push_back({g.points, (int)gi, -1});
        } else {
            for (int i : g.members) {
                const gnss_config &c = e->m[i].cfg;
                units.push_back({(double)c.nx * c.ny * c.nz, -1, i});
            }
        }
    }
    std::stable_sort(units.begin(), units.end(), [](const Unit &a, const Unit &b) { return a.pts > b.pts; });
    std::vector<double> load(e->nbranch, 0.0);
    for (const Unit &u : units) {
        const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        if (u.group >= 0) e->groups[u.group].branch = b;
        else e->m[u.member].branch = b;
        load[b] += u.pts;
    }
}

gnss_status gnss_ensemble_create(const gnss_config *cfgs, int n, int nbranch, gnss_ensemble **out) {
    if (!cfgs || !out || n < 1 || nbranch < 1) return GNSS_ERR_INVALID;
    *out = nullptr;
    const int dev = cfgs[0].device;
    for (int i = 1; i < n; ++i)
        if (cfgs[i].device != dev) return GNSS_ERR_INVALID;   // one device per ensemble
    if (cudaSetDevice(dev) != cudaSuccess) return GNSS_ERR_CUDA;
    gnss_ensemble *e = new gnss_ensemble;
    e->device = dev;
    e->m.resize(n);
    gnss_status st = GNSS_OK;
    for (int i = 0; i < n && st == GNSS_OK; ++i) {
        e->m[i].cfg = cfgs[i];
        st = gnss_create(&cfgs[i], &e->m[i].ctx);
    }
    // groups: members of one geometry, at most GNSS_BATCH_MAX each; batched when the scheme is CN/AB2
    for (int i = 0; i < n && st == GNSS_OK; ++i) {
        Member &mb = e->m[i];
        int gi = -1;
        for (int j = 0; j < (int)e->groups.size(); ++j) {
            const Group &g = e->groups[j];
            if ((int)g.members.size() < GNSS_BATCH_MAX && same_geometry(e->m[g.members[0]].cfg, mb.cfg)) {
                gi = j;
                break;
            }
        }
        if (gi < 0) {
            gi = (int)e->groups.size();
            e->groups.emplace_back();
        }
        e->groups[gi].members.push_back(i);
        mb.group = gi;
    }
    // per group: one buffer of member slots (state + history) and one of scratch slices
    for (size_t gi = 0; gi < e->groups.size() && st == GNSS_OK; ++gi) {
        Group &g = e->groups[gi];
        const gnss_config &c0 = e->m[g.members[0]].cfg;
        const size_t fb = field_bytes_of(c0);
        const int nf = nfields_of(c0);
        const size_t k = g.members.size();
        g.slot = round256(2 * (size_t)nf * fb);
        g.slice = round256(std::max(gnss_scratch_bytes(e->m[g.members[0]].ctx),
                                    gnss_batch_scratch_bytes(e->m[g.members[0]].ctx)));
        g.points = (double)k * c0.nx * c0.ny * c0.nz;
        if (cudaMalloc(&g.buf, k * g.slot) != cudaSuccess || cudaMemset(g.buf, 0, k * g.slot) != cudaSuccess ||
            cudaMalloc(&g.scratch, k * g.slice) != cudaSuccess) {
            cudaGetLastError();
            st = GNSS_ERR_NOMEM;
            break;
        }
        for (size_t j = 0; j < k && st == GNSS_OK; ++j) {
            Member &mb = e->m[g.members[j]];
            mb.buf = static_cast<char *>(g.buf) + j * g.slot;
            mb.state = fields_at(mb.buf, fb, nf);
            mb.hist = fields_at(static_cast<char *>(mb.buf) + nf * fb, fb, nf);
            st = gnss_attach_scratch(mb.ctx, static_cast<char *>(g.scratch) + j * g.slice, g.slice);
        }
    }
    if (st) {
        cudaGetLastError();
        ensemble_free(e);
        return st;
    }
    e->nbranch = std::min(nbranch, n);
    assign_branches(e);
    e->streams.assign(e->nbranch, nullptr);
    e->ev_join.assign(e->nbranch, nullptr);
    for (int b = 0; b < e->nbranch && st == GNSS_OK; ++b) {
        if (cudaStreamCreateWithFlags(&e->streams[b], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->ev_join[b], cudaEventDisableTiming) != cudaSuccess)
            st = GNSS_ERR_CUDA;
    }
    if (!st && (cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking) != cudaSuccess))
        st = GNSS_ERR_CUDA;
    if (st) {
        cudaGetLastError();
        ensemble_free(e);
        return st;
    }
    *out = e;
    return GNSS_OK;
}

gnss_status gnss_ensemble_destroy(gnss_ensemble *e) {
    if (!e) return GNSS_ERR_INVALID;
    ensemble_free(e);
    return GNSS_OK;
}

int gnss_ensemble_size(const gnss_ensemble *e) { return e ? (int)e->m.size() : 0; }

gnss_status gnss_ensemble_member(gnss_ensemble *e, int i, gnss_ctx **ctx, gnss_fields *state, gnss_fields *hist) {
    if (!e || i < 0 || i >= (int)e->m.size()) return GNSS_ERR_INVALID;
    if (ctx) *ctx = e->m[i].ctx;
    if (state) *state = e->m[i].state;
    if (hist) *hist = e->m[i].hist;
    return GNSS_OK;
}

gnss_status gnss_ensemble_upload(gnss_ensemble *e, int i, const void *host_state, void *stream) {
    if (!e || i < 0 || i >= (int)e->m.size() || !host_state) return GNSS_ERR_INVALID;
    if (cudaSetDevice(e->device) != cudaSuccess) return GNSS_ERR_CUDA;
    Member &mb = e->m[i];
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t fb = field_bytes_of(mb.cfg);
    const int nf = nfields_of(mb.cfg);
    if (cudaMemcpyAsync(mb.buf, host_state, nf * fb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(static_cast<char *>(mb.buf) + nf * fb, 0, nf * fb, s) != cudaSuccess)
        return GNSS_ERR_CUDA;
    void *f[5] = {mb.state.u, mb.state.v, mb.state.w, mb.state.s, mb.state.c};
    for (int q = 0; q < nf; ++q) {
        gnss_status st = gnss_dealias(mb.ctx, f[q], stream);
        if (st) return st;
    }
    return GNSS_OK;
}

gnss_status gnss_ensemble_download(gnss_ensemble *e, int i, void *host_state, void *stream) {
    if (!e || i < 0 || i >= (int)e->m.size() || !host_state) return GNSS_ERR_INVALID;
    if (cudaSetDevice(e->device) != cudaSuccess) return GNSS_ERR_CUDA;
    Member &mb = e->m[i];
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t bytes = nfields_of(mb.cfg) * field_bytes_of(mb.cfg);
    if (cudaMemcpyAsync(host_state, mb.buf, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GNSS_ERR_CUDA;
    return GNSS_OK;
}

long long gnss_ensemble_launches_per_step(const gnss_ensemble *e) {
    if (!e) return 0;
    long long s = 0;
    for (const Group &g : e->groups) s += g.launches_per_step;
    return s;
}

// Group g's step as the ensemble runs it: one batched step on the group's
// branch (where its kernels allow), or each member's own step on the member's
// branch.
static gnss_status group_step(gnss_ensemble *e, Group &g, int euler) {
    const Member &m0 = e->m[g.members[0]];
    if (g.batched && gnss_batch_supported(m0.ctx)) {
        gnss_ctx *ctxs[GNSS_BATCH_MAX];
        for (size_t j = 0; j < g.members.size(); ++j) ctxs[j] = e->m[g.members[j]].ctx;
        return gnss_step_batch(ctxs, (int)g.members.size(), &m0.state, &m0.hist, g.slot, g.scratch, g.slice, euler,
                               e->streams[g.branch]);
    }
    for (int i : g.members) {
        Member &mb = e->m[i];
        gnss_status st = gnss_step(mb.ctx, &mb.state, &mb.hist, euler, e->streams[mb.branch]);
        if (st) return st;
    }
    return GNSS_OK;
}

static gnss_status fork_branches(gnss_ensemble *e, cudaStream_t s) {
    if (cudaEventRecord(e->ev_fork, s) != cudaSuccess) return GNSS_ERR_CUDA;
    for (int b = 0; b < e->nbranch; ++b)
        if (cudaStreamWaitEvent(e->streams[b], e->ev_fork, 0) != cudaSuccess) return GNSS_ERR_CUDA;
    return GNSS_OK;
}
static gnss_status join_branches(gnss_ensemble *e, cudaStream_t s) {
    for (int b = 0; b < e->nbranch; ++b) {
        if (cudaEventRecord(e->ev_join[b], e->streams[b]) != cudaSuccess) return GNSS_ERR_CUDA;
        if (cudaStreamWaitEvent(s, e->ev_join[b], 0) != cudaSuccess) return GNSS_ERR_CUDA;
    }
    return GNSS_OK;
}

// Tensor-core passes exist for FP32 x / y lengths 256 and 512.
static bool has_tensor_pass(const gnss_config &c) {
    return c.precision == GNSS_FP32 && (c.nx == 256 || c.nx == 512 || c.ny == 256 || c.ny == 512);
}

// Every group's steps in branch order on the branch streams, forked from and
// joined back into stream `s`: one batched step per group, or the members'
// own steps one after another.
static gnss_status ensemble_issue(gnss_ensemble *e, int n_steps, int euler_first, cudaStream_t s) {
    gnss_status st = fork_branches(e, s);
    if (st) return st;
    for (Group &g : e->groups) {
        for (int k = 0; k < n_steps; ++k) {
            long long l0 = 0, l1 = 0;
            for (int i : g.members) l0 += gnss_launch_count(e->m[i].ctx);
            if ((st = group_step(e, g, (euler_first && k == 0) ? 1 : 0))) return st;
            for (int i : g.members) l1 += gnss_launch_count(e->m[i].ctx);
            g.launches_per_step = l1 - l0;
        }
    }
    return join_branches(e, s);
}

static gnss_status ensemble_capture(gnss_ensemble *e, int n_steps) {
    if (e->gexec) {
        cudaGraphExecDestroy(e->gexec);
        e->gexec = nullptr;
    }
    if (cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeRelaxed) != cudaSuccess) return GNSS_ERR_CUDA;
    gnss_status st = ensemble_issue(e, n_steps, 0, e->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->cap, &g);
    if (st == GNSS_OK && ce != cudaSuccess) st = GNSS_ERR_CUDA;
    if (st == GNSS_OK && cudaGraphInstantiate(&e->gexec, g, 0) != cudaSuccess) st = GNSS_ERR_CUDA;
    if (g) cudaGraphDestroy(g);
    if (st) {
        cudaGetLastError();
        e->gexec = nullptr;
        return st;
    }
    e->g_steps = n_steps;
    return GNSS_OK;
}

gnss_status gnss_ensemble_step(gnss_ensemble *e, int n_steps, void *stream) {
    if (!e || n_steps < 0) return GNSS_ERR_INVALID;
    if (cudaSetDevice(e->device) != cudaSuccess) return GNSS_ERR_CUDA;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n_steps == 0) return GNSS_OK;
    if (e->steps_done == 0) {   // the first step of a run (Euler for the reference scheme), launched directly
        gnss_status st = ensemble_issue(e, 1, 1, s);
        if (st) return st;
        e->steps_done = 1;
        if (--n_steps == 0) return GNSS_OK;
    }
    if (!e->gexec || e->g_steps != n_steps) {
        gnss_status st = ensemble_capture(e, n_steps);
        if (st) return st;
    }
    if (cudaGraphLaunch(e->gexec, s) != cudaSuccess) return GNSS_ERR_CUDA;
    e->steps_done += n_steps;
    return GNSS_OK;
}

gnss_status gnss_ensemble_set_batching(gnss_ensemble *e, int on) {
    if (!e) return GNSS_ERR_INVALID;
    for (Group &g : e->groups) g.batched = on != 0 && gnss_batch_supported(e->m[g.members[0]].ctx);
    assign_branches(e);
    if (e->gexec) {   // the next block of steps is captured anew
        cudaGraphExecDestroy(e->gexec);
        e->gexec = nullptr;
    }
    return GNSS_OK;
}

int gnss_ensemble_batched(const gnss_ensemble *e, int i) {
    if (!e || i < 0 || i >= (int)e->m.size()) return -1;
    const Group &g = e->groups[e->m[i].group];
    return g.batched && gnss_batch_supported(e->m[g.members[0]].ctx) ? 1 : 0;
}

gnss_status gnss_ensemble_autotune(gnss_ensemble *e, int steps, int *choices) {
    if (!e || steps < 1) return GNSS_ERR_INVALID;
    if (cudaSetDevice(e->device) != cudaSuccess) return GNSS_ERR_CUDA;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    gnss_status st = GNSS_OK;
    const int zvariants[3] = {GNSS_VARIANT_REGISTER, GNSS_VARIANT_STAGED, GNSS_VARIANT_WARPSPEC};
    const int pvariants[3] = {GNSS_VARIANT_REGISTER, GNSS_VARIANT_STAGED, GNSS_VARIANT_TENSOR};
    std::vector<int> best(e->groups.size(), GNSS_VARIANT_AUTO);
    std::vector<bool> best_batched(e->groups.size(), false);
    const cudaStream_t ts = e->cap;   // timing stream: the group's steps fork from it and join back
    for (size_t gi = 0; gi < e->groups.size() && !st; ++gi) {
        Group &g = e->groups[gi];
        const Member &m0 = e->m[g.members[0]];
        float tbest = 0.f;
        int vbest = -1;
        bool bbest = false;
        for (int combo = 0; combo < 18 && !st; ++combo) {
            const int zv = zvariants[combo % 3], pv = pvariants[(combo / 3) % 3];
            const bool batched = combo >= 9;   // the same kernels, as one batched launch per stage
            if (pv == GNSS_VARIANT_TENSOR && !has_tensor_pass(m0.cfg)) continue;
            const int v = zv + 4 * pv;   // z variant + 4 * pass variant
            for (int i : g.members)
                if ((st = gnss_set_option(e->m[i].ctx, GNSS_OPT_ZVARIANT, zv)) ||
                    (st = gnss_set_option(e->m[i].ctx, GNSS_OPT_PVARIANT, pv)))
                    break;
            if (st) break;
            int zk = 0;
            if (zv == GNSS_VARIANT_WARPSPEC && (gnss_get_option(m0.ctx, GNSS_OPT_ZKERNEL, &zk) || zk != zv))
                continue;   // no warp-specialised kernel here: the same kernels as the register choice
            if (batched && (g.members.size() < 2 || !gnss_batch_supported(m0.ctx))) continue;
            g.batched = batched;
            if ((st = fork_branches(e, ts)) || (st = group_step(e, g, 1)) || (st = join_branches(e, ts)))
                break;   // warm-up
            cudaEventRecord(t0, ts);
            if ((st = fork_branches(e, ts))) break;
            for (int i = 0; i < steps && !st; ++i) st = group_step(e, g, 0);
            if (st || (st = join_branches(e, ts))) break;
            cudaEventRecord(t1, ts);
            cudaEventSynchronize(t1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            if (vbest < 0 || ms < tbest) {
                tbest = ms;
                vbest = v;
                bbest = batched;
            }
        }
        if (!st) {
            best[gi] = vbest;
            best_batched[gi] = bbest;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st) return st;
    for (size_t gi = 0; gi < e->groups.size(); ++gi) e->groups[gi].batched = best_batched[gi];
    for (size_t i = 0; i < e->m.size(); ++i) {
        Member &mb = e->m[i];
        const int v = best[mb.group];
        if ((st = gnss_set_option(mb.ctx, GNSS_OPT_ZVARIANT, v & 3)) ||
            (st = gnss_set_option(mb.ctx, GNSS_OPT_PVARIANT, v >> 2)))
            return st;
        if (choices) choices[i] = v;
        const size_t fb = field_bytes_of(mb.cfg);
        if (cudaMemset(mb.buf, 0, 2 * nfields_of(mb.cfg) * fb) != cudaSuccess) return GNSS_ERR_CUDA;
    }
    assign_branches(e);
    if (cudaDeviceSynchronize() != cudaSuccess) return GNSS_ERR_CUDA;
    if (e->gexec) {
        cudaGraphExecDestroy(e->gexec);
        e->gexec = nullptr;
    }
    e->steps_done = 0;
    return GNSS_OK;
}

// ====================================================================== server
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    gnss_config cfg{};
    int n_steps = 0;
    size_t state_bytes = 0, reserve = 0, scratch_bytes = 0;
    void *h_in = nullptr, *h_out = nullptr;   // pinned
    double stats[GNSS_NSTATS] = {};
    double t_submit = 0, t_admit = 0, t_done = 0;
    gnss_status status = GNSS_OK;
    gnss_ctx *ctx = nullptr;
    void *dev = nullptr, *scratch = nullptr;
    gnss_fields state{}, hist{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int steps_issued = 0;
    int phase = 0;   // 0 queued, 1 stepping, 2 copying out, 3 ended
};

}  // namespace

// Pinned host buffers, reused across requests (page-locking is slow, so a
// steady stream of requests allocates none).
struct PinnedPool {
    std::mutex mu;
    std::multimap<size_t, void *> free_;
    std::vector<void *> all;
    void *get(size_t bytes) {
        {
            std::lock_guard<std::mutex> lk(mu);
            auto it = free_.lower_bound(bytes);
            if (it != free_.end() && it->first <= 2 * bytes) {
                void *p = it->second;
                free_.erase(it);
                return p;
            }
        }
        void *p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        std::lock_guard<std::mutex> lk(mu);
        all.push_back(p);
        sizes[p] = bytes;
        return p;
    }
    void put(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu);
        free_.emplace(sizes[p], p);
    }
    ~PinnedPool() {
        for (void *p : all) cudaFreeHost(p);
    }
    std::map<void *, size_t> sizes;
};

struct gnss_server {
    gnss_server_config cfg{};
    PinnedPool pinned;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::vector<Request *> active;            // scheduler thread only (sizes read under mu)
    std::map<long long, Request *> reqs;      // every request not yet fetched
    std::vector<gnss_ctx *> retired;          // contexts of ended requests, destroyed with the server
    long long next_id = 1;
    bool stop = false;
    gnss_server_report rep{};
    Clock::time_point t0;
    std::thread th;
};

static double now_s(const gnss_server *s) {
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

static void req_release_device(gnss_server *s, Request *r) {
    if (r->gexec) {
        cudaGraphExecDestroy(r->gexec);
        r->gexec = nullptr;
    }
    if (r->dev) cudaFreeAsync(r->dev, r->stream);
    if (r->scratch) cudaFreeAsync(r->scratch, r->stream);
    r->dev = r->scratch = nullptr;
    if (r->ev) cudaEventDestroy(r->ev);
    if (r->stream) cudaStreamDestroy(r->stream);   // returns at once; pending frees still run
    r->ev = nullptr;
    r->stream = nullptr;
    if (r->ctx) s->retired.push_back(r->ctx);
    r->ctx = nullptr;
}

// Upload, dealias and the first step.  Runs on the scheduler thread.
static gnss_status req_start(Request *r) {
    const int nf = nfields_of(r->cfg);
    const size_t fb = field_bytes_of(r->cfg);
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess)
        return GNSS_ERR_CUDA;
    if (cudaMallocAsync(&r->dev, 2 * nf * fb, r->stream) != cudaSuccess ||
        cudaMallocAsync(&r->scratch, r->scratch_bytes, r->stream) != cudaSuccess) {
        cudaGetLastError();
        return GNSS_ERR_NOMEM;
    }
    r->state = fields_at(r->dev, fb, nf);
    r->hist = fields_at(static_cast<char *>(r->dev) + nf * fb, fb, nf);
    gnss_status st = gnss_attach_scratch(r->ctx, r->scratch, r->scratch_bytes);
    if (st) return st;
    if (cudaMemcpyAsync(r->dev, r->h_in, r->state_bytes, cudaMemcpyHostToDevice, r->stream) != cudaSuccess ||
        cudaMemsetAsync(static_cast<char *>(r->dev) + nf * fb, 0, nf * fb, r->stream) != cudaSuccess)
        return GNSS_ERR_CUDA;
    void *f[5] = {r->state.u, r->state.v, r->state.w, r->state.s, r->state.c};
    for (int q = 0; q < nf; ++q)
        if ((st = gnss_dealias(r->ctx, f[q], r->stream))) return st;   // as gnss_run_host (main.cu:156)
    if (r->n_steps > 0) {
        if ((st = gnss_step(r->ctx, &r->state, &r->hist, 1, r->stream))) return st;
        r->steps_issued = 1;
    }
    if (cudaEventRecord(r->ev, r->stream) != cudaSuccess) return GNSS_ERR_CUDA;
    return GNSS_OK;
}

static gnss_status req_chunk(const gnss_server *s, Request *r) {
    const int spl = std::max(1, s->cfg.steps_per_launch);
    const int k = std::min(spl, r->n_steps - r->steps_issued);
    gnss_status st = GNSS_OK;
    if (k == spl && spl > 1) {
        if (!r->gexec) {   // capture once per request, replay for every full chunk
            if (cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) return GNSS_ERR_CUDA;
            for (int i = 0; i < k && !st; ++i) st = gnss_step(r->ctx, &r->state, &r->hist, 0, r->stream);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(r->stream, &g);
            if (!st && ce != cudaSuccess) st = GNSS_ERR_CUDA;
            if (!st && cudaGraphInstantiate(&r->gexec, g, 0) != cudaSuccess) st = GNSS_ERR_CUDA;
            if (g) cudaGraphDestroy(g);
            if (st) {
                cudaGetLastError();
                r->gexec = nullptr;
                return st;
            }
        }
        if (cudaGraphLaunch(r->gexec, r->stream) != cudaSuccess) return GNSS_ERR_CUDA;
    } else {
        for (int i = 0; i < k && !st; ++i) st = gnss_step(r->ctx, &r->state, &r->hist, 0, r->stream);
        if (st) return st;
    }
    r->steps_issued += k;
    return cudaEventRecord(r->ev, r->stream) == cudaSuccess ? GNSS_OK : GNSS_ERR_CUDA;
}

static gnss_status req_finish(Request *r) {
    gnss_status st = gnss_stats(r->ctx, &r->state, r->stats, r->stream);   // the stream is idle here
    if (st) return st;
    if (cudaMemcpyAsync(r->h_out, r->dev, r->state_bytes, cudaMemcpyDeviceToHost, r->stream) != cudaSuccess ||
        cudaEventRecord(r->ev, r->stream) != cudaSuccess)
        return GNSS_ERR_CUDA;
    return GNSS_OK;
}

static void server_loop(gnss_server *s) {
    cudaSetDevice(s->cfg.device);
    double busy_start = -1.0;
    for (;;) {
        std::vector<Request *> admit;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->active.empty() && (s->pending.empty() || s->stop)) {
                if (busy_start >= 0) {
                    s->rep.busy_seconds += now_s(s) - busy_start;
                    busy_start = -1.0;
                }
                if (s->stop) break;
                s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
                continue;
            }
            // admission in arrival order: the head waits until it fits
            while (!s->stop && !s->pending.empty() &&
                   (int)(s->active.size() + admit.size()) < std::max(1, s->cfg.max_active)) {
                Request *r = s->pending.front();
                if (s->rep.bytes_reserved + r->reserve > s->cfg.budget_bytes) {
                    if (s->active.empty() && admit.empty()) {   // can never fit
                        s->pending.pop_front();
                        r->status = GNSS_ERR_NOMEM;
                        r->phase = 3;
                        r->t_done = now_s(s);
                        s->rep.failed++;
                        s->cv_done.notify_all();
                        continue;
                    }
                    break;
                }
                s->pending.pop_front();
                s->rep.bytes_reserved += r->reserve;
                s->rep.bytes_reserved_max = std::max(s->rep.bytes_reserved_max, s->rep.bytes_reserved);
                s->rep.admitted++;
                admit.push_back(r);
            }
        }
        bool progress = !admit.empty();
        for (Request *r : admit) {
            r->t_admit = now_s(s);
            r->phase = 1;
            r->status = req_start(r);
            std::lock_guard<std::mutex> lk(s->mu);
            s->active.push_back(r);
            s->rep.active_max = std::max(s->rep.active_max, (int)s->active.size());
        }
        if (!s->active.empty() && busy_start < 0) busy_start = now_s(s);
        for (size_t i = 0; i < s->active.size();) {
            Request *r = s->active[i];
            if (r->status == GNSS_OK && r->ev) {
                const cudaError_t q = cudaEventQuery(r->ev);
                if (q == cudaErrorNotReady) {
                    ++i;
                    continue;
                }
                if (q != cudaSuccess) r->status = GNSS_ERR_CUDA;
            }
            progress = true;
            if (r->status == GNSS_OK && r->phase == 1) {
                if (r->steps_issued < r->n_steps) {
                    r->status = req_chunk(s, r);
                } else {   // every step has run: statistics and copy-out
                    r->status = req_finish(r);
                    std::lock_guard<std::mutex> lk(s->mu);
                    if (r->status == GNSS_OK) r->phase = 2;
                }
            }
            ++i;
        }
        // requests whose copy-out completed (phase 2), or that failed, end here
        for (size_t i = 0; i < s->active.size();) {
            Request *r = s->active[i];
            const bool done = r->status != GNSS_OK || (r->phase == 2 && cudaEventQuery(r->ev) == cudaSuccess);
            if (!done) {
                ++i;
                continue;
            }
            progress = true;
            req_release_device(s, r);
            std::lock_guard<std::mutex> lk(s->mu);
            r->t_done = now_s(s);
            r->phase = 3;
            s->rep.bytes_reserved -= r->reserve;
            if (r->status == GNSS_OK) {
                s->rep.completed++;
                s->rep.point_steps += (double)r->cfg.nx * r->cfg.ny * r->cfg.nz * r->n_steps;
            } else {
                s->rep.failed++;
            }
            s->active.erase(s->active.begin() + (long)i);
            s->cv_done.notify_all();
        }
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

gnss_status gnss_server_create(const gnss_server_config *cfg, gnss_server **out) {
    if (!cfg || !out || cfg->max_active < 1 || cfg->steps_per_launch < 1) return GNSS_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
        cudaGetLastError();
        return GNSS_ERR_CUDA;
    }
    gnss_server *s = new gnss_server;
    s->cfg = *cfg;
    s->t0 = Clock::now();
    s->th = std::thread(server_loop, s);
    *out = s;
    return GNSS_OK;
}

gnss_status gnss_server_destroy(gnss_server *s) {
    if (!s) return GNSS_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (Request *r : s->pending) {   // dropped
            r->status = GNSS_ERR_INVALID;
            r->phase = 3;
        }
        s->pending.clear();
    }
    s->cv_work.notify_all();
    s->th.join();
    cudaSetDevice(s->cfg.device);
    cudaDeviceSynchronize();
    for (gnss_ctx *c : s->retired) gnss_destroy(c);
    for (auto &kv : s->reqs) {
        Request *r = kv.second;
        if (r->ctx) gnss_destroy(r->ctx);
        delete r;   // pinned buffers go with the pool
    }
    delete s;
    return GNSS_OK;
}

gnss_status gnss_server_submit(gnss_server *s, const gnss_config *cfg, const void *host_state, int n_steps,
                               long long *id) {
    if (!s || !cfg || !host_state || n_steps < 0) return GNSS_ERR_INVALID;
    if (cfg->device != s->cfg.device) return GNSS_ERR_INVALID;
    const double t_entry = now_s(s);
    Request *r = new Request;
    r->cfg = *cfg;
    r->n_steps = n_steps;
    gnss_status st = gnss_create(cfg, &r->ctx);
    if (st) {
        delete r;
        return st;
    }
    const int nf = nfields_of(*cfg);
    const size_t fb = field_bytes_of(*cfg);
    r->state_bytes = nf * fb;
    r->scratch_bytes = round256(gnss_scratch_bytes(r->ctx));
    r->reserve = 2 * nf * fb + r->scratch_bytes + gnss_workspace_bytes(r->ctx);
    r->h_in = s->pinned.get(r->state_bytes);
    r->h_out = s->pinned.get(r->state_bytes);
    if (!r->h_in || !r->h_out) {
        s->pinned.put(r->h_in);
        s->pinned.put(r->h_out);
        gnss_destroy(r->ctx);
        delete r;
        return GNSS_ERR_NOMEM;
    }
    std::memcpy(r->h_in, host_state, r->state_bytes);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            s->pinned.put(r->h_in);
            s->pinned.put(r->h_out);
            gnss_destroy(r->ctx);
            delete r;
            return GNSS_ERR_INVALID;
        }
        r->id = s->next_id++;
        r->t_submit = t_entry;   // latency counts the submission's own copy
        s->reqs[r->id] = r;
        s->pending.push_back(r);
        s->rep.submitted++;
    }
    s->cv_work.notify_one();
    if (id) *id = r->id;
    return GNSS_OK;
}

gnss_status gnss_server_wait(gnss_server *s, long long id, double timeout_s) {
    if (!s) return GNSS_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return GNSS_ERR_INVALID;
    Request *r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->phase == 3; });
    return ok ? GNSS_OK : GNSS_ERR_TIMEOUT;
}

gnss_status gnss_server_result(gnss_server *s, long long id, void *host_state_out, double *stats, double *times) {
    if (!s) return GNSS_ERR_INVALID;
    Request *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end() || it->second->phase != 3) return GNSS_ERR_INVALID;
        r = it->second;
        s->reqs.erase(it);
    }
    const gnss_status st = r->status;
    if (st == GNSS_OK) {
        if (host_state_out) std::memcpy(host_state_out, r->h_out, r->state_bytes);
        if (stats) std::memcpy(stats, r->stats, sizeof r->stats);
    }
    if (times) {
        times[0] = r->t_submit;
        times[1] = r->t_admit;
        times[2] = r->t_done;
    }
    if (r->ctx) gnss_destroy(r->ctx);   // never admitted
    s->pinned.put(r->h_in);
    s->pinned.put(r->h_out);
    delete r;
    return st;
}

gnss_status gnss_server_report_get(gnss_server *s, gnss_server_report *out) {
    if (!s || !out) return GNSS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->rep;
    return GNSS_OK;
}
