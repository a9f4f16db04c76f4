// batch_host.cu — batched evaluation of many models over the resident points
// (lcg_light_curve_batch_resident).
//
// The MCMC and Levenberg-Marquardt callers evaluate light_curve_comp for
// many parameter vectors over one data set (mcmc_solver.cpp:1062-1070,
// levmarq_solver.cpp:789-886). One model's grids keep a B200 busy only at
// the largest resolutions, so here all models of a batch go through every
// stage together:
//   * layout: the two star grids of model m are slots 2m and 2m+1; their
//     faces are concatenated in one set of point arrays, their flat records
//     start at multiples of 1024 faces, and their flux work is a list of
//     (chunk, phase tile) CTAs over all slots;
//   * the ring tables of grids without infill depend on nlat alone and are
//     computed once per nlat (set_star_grid.cpp:241-320, numface.cpp);
//   * per call, only the slots whose geometry (GeomKey) changed go through
//     grid + eclipse, and only those whose continuum (ContKey) changed
//     through continuum + partition (the per-model form of the exact-reuse
//     cache, light_curve_comp.cpp:34-117);
//   * the work lists and per-model parameters are one host table copied in
//     one transfer, and the whole sequence is one CUDA graph, captured once
//     per layout and replayed.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "context.h"

namespace lcg {
namespace eng {

namespace {

constexpr int64_t kSlotAlign = 1024;  // flat records and partition blocks

struct RingSet {
    int32_t ring0, nrings;
    int64_t nface, ntiled, nhalf;  // numface, the tiling's faces, half-faces
};

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Host threads kept for the per-model setup of batch calls (started on first
// use): spawning them per call cost more than the setup of a few dozen
// models. One job at a time (calls from several host threads queue on
// call_mu); the caller works on the job too, so it finishes even before the
// workers wake.
class SetupPool {
public:
    static SetupPool &get() {
        static SetupPool p;
        return p;
    }
    int threads() const { return (int)th_.size() + 1; }

    void run(int n, const std::function<void(int)> &f) {
        std::lock_guard<std::mutex> call(call_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &f;
            n_ = n;
            next_.store(0);
            busy_ = (int)th_.size();
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return busy_ == 0; });
        job_ = nullptr;
    }

private:
    SetupPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nt = (int)std::min<unsigned>(15u, hw > 1 ? hw - 1 : 0u);
        for (int t = 0; t < nt; t++) th_.emplace_back([this] { loop(); });
    }
    ~SetupPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            gen_++;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void work() {
        for (int i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*job_)(i);
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> lk(mu_);
            if (--busy_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_, call_mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)> *job_ = nullptr;
    int n_ = 0, busy_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
    std::atomic<int> next_{0};
};

// Runs f(i) for i in [0, n): inline for a few items, else on SetupPool.
template <class F>
void parallel_for(int n, F f) {
    if (n < 8) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    const std::function<void(int)> g = f;
    SetupPool::get().run(n, g);
}

}  // namespace

struct BatchState {
    // layout key
    int32_t nmodels = -1, n = 0, flags = 0, want_calc = 0;
    int64_t nent = 0;
    const void *data_p = nullptr;
    std::vector<int32_t> nlat;  // nlat1f, nlat2f per model
    // layout
    int32_t nslots = 0;
    int64_t nfaces = 0, nflat = 0, nblk = 0, ldp = 0;
    FluxPlan plan{};
    bool tuned = false;      // the flux plan was chosen by autotune_flux
    DBuf<int64_t> tune_pre;  // chunk offsets of a candidate plan while timing
    std::vector<int64_t> face0, flat0, blk0, chunk_pre;
    std::vector<RingSet> slot_rings;
    // ring pool, one table per nlat
    std::map<int32_t, RingSet> ringsets;
    std::vector<RingRec> h_rings;
    DBuf<RingRec> rings;
    // per-model exact-reuse keys: the last model evaluated in each position,
    // its input scale and the data version its results belong to
    std::vector<lcg_model> key;
    std::vector<uint8_t> key_ok;
    std::vector<double> key_sfac0;
    int64_t data_version = -1;
    // host table (pinned) and its device copy
    unsigned char *h_tab = nullptr;
    size_t tab_bytes = 0;
    DBuf<unsigned char> d_tab;
    size_t o_slots = 0, o_models = 0, o_face0 = 0, o_chunk = 0, o_counts = 0, o_geo_slot = 0,
           o_geo_half = 0, o_geo_face = 0, o_cont_slot = 0, o_cont_face = 0, o_cont_blk = 0;
    // device arrays
    DBuf<double> px, py, pz, nx, ny, nz, ein, eout;
    DBuf<float> area, grav, flux, fp;
    DBuf<uint8_t> necl;
    DBuf<ulonglong2> ecl;
    DBuf<int64_t> n0;
    DBuf<int32_t> blockcnt, queue, counters;
    DBuf<DevStatus> st;
    DBuf<float4> ef, runb;
    DBuf<ulonglong2> runh;
    DBuf<unsigned long long> pfx;
    DBuf<double4> es;
    DBuf<int32_t> hits;
    DBuf<double> w1, w2, part, osum, calc, sfac, out;
    // results (pinned): calc, sfac, out, status
    unsigned char *h_res = nullptr;
    size_t res_bytes = 0, r_calc = 0, r_sfac = 0, r_out = 0, r_st = 0;
    cudaGraphExec_t exec = nullptr;
    int64_t graph_kernels = 0;  // kernels per graph launch
    // lcg_batch_curves: selected rows gathered on the device, then one copy
    DBuf<int32_t> rows;
    DBuf<double> gathered;
    double *h_rows = nullptr;
    size_t h_rows_cap = 0;

    template <class T>
    T *tab(size_t off) { return reinterpret_cast<T *>(h_tab + off); }
    template <class T>
    T *res(size_t off) { return reinterpret_cast<T *>(h_res + off); }

    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    void free_all() {
        drop_graph();
        DBuf<double> *d[] = {&px, &py, &pz, &nx, &ny, &nz, &ein, &eout,
                             &w1, &w2, &part, &osum, &calc, &sfac, &out};
        for (auto *b : d) b->release();
        area.release(); grav.release(); flux.release(); fp.release(); necl.release();
        ecl.release(); n0.release(); blockcnt.release(); queue.release(); counters.release();
        st.release(); ef.release(); pfx.release(); runb.release(); runh.release(); rings.release(); es.release(); hits.release(); d_tab.release();
        rows.release(); gathered.release(); tune_pre.release();
        if (h_rows) cudaFreeHost(h_rows);
        h_rows = nullptr;
        h_rows_cap = 0;
        if (h_tab) cudaFreeHost(h_tab);
        if (h_res) cudaFreeHost(h_res);
        h_tab = h_res = nullptr;
    }

    BatchDev dev() {
        BatchDev b{};
        unsigned char *d = d_tab.p;
        b.slots = reinterpret_cast<const SlotDev *>(d + o_slots);
        b.models = reinterpret_cast<const ModelDev *>(d + o_models);
        b.face0 = reinterpret_cast<const int64_t *>(d + o_face0);
        b.chunk_pre = reinterpret_cast<const int64_t *>(d + o_chunk);
        b.rings = rings.p;
        b.nslots = nslots;
        b.nmodels = nmodels;
        b.g = GridDev{px.p, py.p, pz.p, nx.p, ny.p, nz.p, area.p, grav.p, flux.p,
                      necl.p, ein.p, eout.p, nfaces};
        b.fp = fp.p;
        b.runb = runb.p;
        b.runh = runh.p;
        b.ecl = ecl.p;
        b.n0 = n0.p;
        b.blockcnt = blockcnt.p;
        b.queue = queue.p;
        b.qcap = nfaces;
        b.counters = counters.p;
        b.es = es.p;
        b.hits = hits.p;
        b.st = st.p;
        b.counts = reinterpret_cast<const int32_t *>(d + o_counts);
        b.geo_slot = reinterpret_cast<const int32_t *>(d + o_geo_slot);
        b.geo_half = reinterpret_cast<const int64_t *>(d + o_geo_half);
        b.geo_face = reinterpret_cast<const int64_t *>(d + o_geo_face);
        b.cont_slot = reinterpret_cast<const int32_t *>(d + o_cont_slot);
        b.cont_face = reinterpret_cast<const int64_t *>(d + o_cont_face);
        b.cont_blk = reinterpret_cast<const int64_t *>(d + o_cont_blk);
        return b;
    }
    BatchPhases phases() { return BatchPhases{ef.p, w1.p, w2.p, ldp, nent, pfx.p}; }
};

void batch_release(BatchState *b) {
    if (!b) return;
    b->free_all();
    delete b;
}

namespace {

// Face count and ring table of a grid without infill (numface.cpp:14-52,
// set_star_grid.cpp:241-320), added to the pool once per nlat.
void ring_set(BatchState &B, int32_t nlat, RingSet &out) {
    auto it = B.ringsets.find(nlat);
    if (it != B.ringsets.end()) {
        out = it->second;
        return;
    }
    StarSetup s{};
    s.nhalf = 0;
    int nface = 0;
    add_rings(kStar1, s, nface, 0., kPi, kPi / nlat, 0, 0);
    RingSet r{(int32_t)B.h_rings.size(), (int32_t)s.rings.size(),
              numface(nlat, false, 0., 0., 0, 0), nface, s.nhalf};
    B.h_rings.insert(B.h_rings.end(), s.rings.begin(), s.rings.end());
    B.ringsets[nlat] = r;
    out = r;
}

// Lays out slots, records, flux chunks and the host table for a batch of
// nmodels with the given grid resolutions, and (re)allocates everything.
lcg_status relayout(lcg_ctx *c, BatchState &B, const lcg_model *models, int32_t nmodels,
                    int32_t flags, int want_calc) {
    B.drop_graph();
    B.tuned = false;
    B.nmodels = nmodels;
    B.n = c->data_n;
    B.nent = c->data_nent;
    B.data_p = c->data.p;
    B.flags = flags;
    B.want_calc = want_calc;
    B.nslots = 2 * nmodels;
    B.nlat.resize(2 * (size_t)nmodels);
    B.slot_rings.resize(B.nslots);
    B.face0.assign(B.nslots + 1, 0);
    B.flat0.assign(B.nslots + 1, 0);
    B.blk0.assign(B.nslots + 1, 0);
    B.chunk_pre.assign(B.nslots + 1, 0);
    const size_t nring_before = B.h_rings.size();
    for (int32_t m = 0; m < nmodels; m++) {
        B.nlat[2 * m] = models[m].nlat1f;
        B.nlat[2 * m + 1] = models[m].nlat2f;
        for (int k = 0; k < 2; k++) {
            const int s = 2 * m + k;
            RingSet r;
            ring_set(B, B.nlat[s], r);
            B.slot_rings[s] = r;
            B.face0[s + 1] = B.face0[s] + r.nface;
            B.flat0[s + 1] = B.flat0[s] + (int64_t)align_up((size_t)r.nface, kSlotAlign);
            B.blk0[s + 1] = B.blk0[s] + (r.nface + kSlotAlign - 1) / kSlotAlign;
        }
    }
    B.nfaces = B.face0[B.nslots];
    B.nflat = B.flat0[B.nslots];
    B.nblk = B.blk0[B.nslots];
    if (B.nfaces >= (int64_t)0x7fffffff)
        return c->fail(LCG_E_CAPACITY, "batch: %lld faces exceed the 2^31 face index",
                       (long long)B.nfaces);
    // flux plan: the single-grid plan for entries per thread and phase tiles;
    // then the largest chunk (dividing 1024) that still fills the SMs
    B.plan = plan_flux(1, 1, B.nfaces, B.nent, c->nsm);
    int64_t chunk = 1024, total = 0;
    const int64_t want = (int64_t)c->nsm * 4;
    for (;;) {
        total = 0;
        for (int s = 0; s < B.nslots; s++)
            total += (B.slot_rings[s].nface + chunk - 1) / chunk;
        if (chunk <= 64 || total * B.plan.ntile >= want) break;
        chunk >>= 1;
    }
    B.plan.chunk = chunk;
    B.plan.nchunk = total;
    if (total * B.plan.ntile >= (int64_t)0x7fffffff)
        return c->fail(LCG_E_CAPACITY, "batch: too many flux tiles");
    for (int s = 0; s < B.nslots; s++)
        B.chunk_pre[s + 1] = B.chunk_pre[s] + (B.slot_rings[s].nface + chunk - 1) / chunk;
    B.ldp = ((B.nent + 3) / 4) * 4;

    // host table sections
    size_t o = 0;
    auto sect = [&](size_t bytes) {
        const size_t at = o;
        o = align_up(o + bytes, 256);
        return at;
    };
    const size_t ns = (size_t)B.nslots;
    B.o_slots = sect(ns * sizeof(SlotDev));
    B.o_models = sect((size_t)nmodels * sizeof(ModelDev));
    B.o_face0 = sect((ns + 1) * 8);
    B.o_chunk = sect((ns + 1) * 8);
    B.o_counts = sect(8);
    B.o_geo_slot = sect(ns * 4);
    B.o_geo_half = sect((ns + 1) * 8);
    B.o_geo_face = sect((ns + 1) * 8);
    B.o_cont_slot = sect(ns * 4);
    B.o_cont_face = sect((ns + 1) * 8);
    B.o_cont_blk = sect((ns + 1) * 8);
    B.tab_bytes = o;
    if (B.h_tab) cudaFreeHost(B.h_tab);
    B.h_tab = nullptr;
    cudaError_t e;
    if ((e = cudaHostAlloc((void **)&B.h_tab, B.tab_bytes, cudaHostAllocDefault)))
        return c->cuda_fail(e, "batch table");
    memset(B.h_tab, 0, B.tab_bytes);
    memcpy(B.tab<int64_t>(B.o_face0), B.face0.data(), (ns + 1) * 8);
    memcpy(B.tab<int64_t>(B.o_chunk), B.chunk_pre.data(), (ns + 1) * 8);

    // results
    const size_t nm = (size_t)nmodels;
    o = 0;
    B.r_calc = sect(want_calc ? nm * (size_t)B.n * 8 : 0);
    B.r_sfac = sect(nm * 5 * 8);
    B.r_out = sect(nm * 3 * 8);
    B.r_st = sect(nm * sizeof(DevStatus));
    B.res_bytes = o;
    if (B.h_res) cudaFreeHost(B.h_res);
    B.h_res = nullptr;
    if ((e = cudaHostAlloc((void **)&B.h_res, B.res_bytes, cudaHostAllocDefault)))
        return c->cuda_fail(e, "batch results");

    // device arrays
    const size_t nf = (size_t)B.nfaces;
    DBuf<double> *d[] = {&B.px, &B.py, &B.pz, &B.nx, &B.ny, &B.nz, &B.ein, &B.eout};
    for (auto *b : d)
        if ((e = b->ensure(nf))) return c->cuda_fail(e, "batch grids");
    if ((e = B.area.ensure(nf)) || (e = B.grav.ensure(nf)) || (e = B.flux.ensure(nf)) ||
        (e = B.necl.ensure(nf)) || (e = B.queue.ensure(nf)) ||
        (e = B.fp.ensure(8 * (size_t)B.nflat)) || (e = B.ecl.ensure((size_t)B.nflat)) ||
        (e = B.runb.ensure((size_t)B.nflat / 64)) || (e = B.runh.ensure((size_t)B.nflat / 64)) ||
        (e = B.n0.ensure(ns)) || (e = B.blockcnt.ensure((size_t)B.nblk)) ||
        (e = B.counters.ensure(8)) || (e = B.st.ensure(nm)) ||
        (e = B.es.ensure(nf)) || (e = B.hits.ensure(nf)) ||
        (e = B.ef.ensure(nm * (size_t)B.ldp)) || (e = B.pfx.ensure(nm * (size_t)B.ldp)) || (e = B.w1.ensure(nm * (size_t)B.ldp)) ||
        (e = B.w2.ensure(nm * (size_t)B.ldp)) ||
        (e = B.part.ensure((size_t)std::max<int64_t>(B.plan.nchunk, 1) * (size_t)B.ldp)) ||
        (e = B.osum.ensure(ns * (size_t)B.ldp)) || (e = B.calc.ensure(nm * (size_t)B.n)) ||
        (e = B.sfac.ensure(nm * 5)) || (e = B.out.ensure(nm * 3)) ||
        (e = B.d_tab.ensure(B.tab_bytes)))
        return c->cuda_fail(e, "batch buffers");
    if (B.h_rings.size() != nring_before || !B.rings.p) {
        if ((e = B.rings.ensure(B.h_rings.size()))) return c->cuda_fail(e, "ring pool");
        cudaMemcpyAsync(B.rings.p, B.h_rings.data(), B.h_rings.size() * sizeof(RingRec),
                        cudaMemcpyHostToDevice, c->stream);
    }
    // an odd pad record or a never-built slot must read as zeros
    cudaMemsetAsync(B.fp.p, 0, 8 * (size_t)B.nflat * sizeof(float), c->stream);
    cudaMemsetAsync(B.ecl.p, 0, (size_t)B.nflat * sizeof(ulonglong2), c->stream);
    cudaMemsetAsync(B.runb.p, 0, (size_t)B.nflat / 64 * sizeof(float4), c->stream);
    cudaMemsetAsync(B.runh.p, 0, (size_t)B.nflat / 64 * sizeof(ulonglong2), c->stream);
    cudaMemsetAsync(B.n0.p, 0, ns * sizeof(int64_t), c->stream);
    B.key.assign(nm, lcg_model{});
    B.key_ok.assign(nm, 0);
    B.key_sfac0.assign(nm, 0.);
    for (int s = 0; s < B.nslots; s++) {
        SlotDev &S = B.tab<SlotDev>(B.o_slots)[s];
        S.face0 = B.face0[s];
        S.nface = B.slot_rings[s].nface;
        S.ntiled = B.slot_rings[s].ntiled;
        S.flat0 = B.flat0[s];
        S.blk0 = B.blk0[s];
        S.ring0 = B.slot_rings[s].ring0;
        S.model = s / 2;
    }
    return LCG_OK;
}

bool same_layout(const BatchState &B, const lcg_ctx *c, const lcg_model *models,
                 int32_t nmodels, int32_t flags, int want_calc) {
    if (B.nmodels != nmodels || B.n != c->data_n || B.nent != c->data_nent ||
        B.data_p != (const void *)c->data.p || B.flags != flags || B.want_calc != want_calc)
        return false;
    for (int32_t m = 0; m < nmodels; m++)
        if (B.nlat[2 * m] != models[m].nlat1f || B.nlat[2 * m + 1] != models[m].nlat2f)
            return false;
    return true;
}

// Models the batched path covers: the fast mixed sweep applies to both stars
// and each star has a single grid (coarse = fine, no infill).
// Models the batched stages cover; the others (beaming, lensing, limb cut-off,
// coarse grids, infill, disc / spot / iscale models) go one by one through the
// single-model path.
bool batchable(const lcg_model &m) {
    return !m.add_disc && !m.add_spot && !m.iscale &&
           m.beam_factor1 == 0. && m.beam_factor2 == 0. && !m.glens1 && m.mucrit1 <= 0. &&
           m.mucrit2 <= 0. && m.nlat1c == m.nlat1f && m.nlat2c == m.nlat2f &&
           (!m.npole || (m.nlatfill == 0 && m.nlngfill == 0));
}

// Flux-plan autotuner. On the first call of a layout, once the stages before
// the sweep have built the records and phases, each candidate plan (phase
// entries per thread 4, 2 or 1; face chunks of 1024, 512, 256 or 128 faces) times
// the batched sweep on them (one warm-up launch, then the mean of two timed
// ones) and the fastest becomes the layout's plan for that call and every
// later one (the captured graph included). The choice is kept per layout
// (slot face counts, phase entries, SM count) for the whole process, so every
// context evaluating that layout sums in the same chunks and gives the same
// results; a new process measures again.
struct PlanChoice {
    int ppt;
    int64_t chunk;
};
std::mutex g_plan_mu;
std::map<std::vector<int64_t>, PlanChoice> g_plans;

FluxPlan plan_for(const BatchState &B, int ppt, int64_t chunk, std::vector<int64_t> &pre) {
    FluxPlan p = B.plan;
    p.ppt = ppt;
    p.chunk = chunk;
    p.ntile = (B.nent + (int64_t)256 * ppt - 1) / ((int64_t)256 * ppt);
    pre.assign((size_t)B.nslots + 1, 0);
    for (int sl = 0; sl < B.nslots; sl++)
        pre[sl + 1] = pre[sl] + (B.slot_rings[sl].nface + chunk - 1) / chunk;
    p.nchunk = pre[B.nslots];
    return p;
}

cudaError_t autotune_flux(lcg_ctx *c, BatchState &B) {
    cudaStream_t s = c->stream;
    cudaError_t e;
    std::vector<int64_t> key = {B.nent, (int64_t)c->nsm, (int64_t)B.nslots};
    for (int sl = 0; sl < B.nslots; sl++) key.push_back(B.slot_rings[sl].nface);
    PlanChoice choice{0, 0};
    {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        auto it = g_plans.find(key);
        if (it != g_plans.end()) choice = it->second;
    }
    if (!choice.ppt) {
        const int ppts[] = {4, 2, 1};
        const int64_t chunks[] = {1024, 512, 256, 128};
        std::vector<FluxPlan> plans;
        std::vector<std::vector<int64_t>> pres;
        int64_t most = 0;
        for (int64_t ch : chunks)
            for (int ppt : ppts) {
                std::vector<int64_t> pre;
                FluxPlan p = plan_for(B, ppt, ch, pre);
                if (p.nchunk * p.ntile >= (int64_t)0x7fffffff) continue;
                most = std::max(most, p.nchunk);
                plans.push_back(p);
                pres.push_back(std::move(pre));
            }
        if (plans.empty()) return cudaSuccess;
        if ((e = B.part.ensure((size_t)std::max<int64_t>(most, 1) * (size_t)B.ldp)) ||
            (e = B.tune_pre.ensure((size_t)B.nslots + 1)))
            return e;
        cudaEvent_t ev0, ev1;
        if ((e = cudaEventCreate(&ev0))) return e;
        if ((e = cudaEventCreate(&ev1))) {
            cudaEventDestroy(ev0);
            return e;
        }
        const BatchPhases ph = B.phases();
        double best = 1e300;
        size_t pick = 0;
        for (size_t i = 0; i < plans.size(); i++) {
            cudaMemcpyAsync(B.tune_pre.p, pres[i].data(), pres[i].size() * sizeof(int64_t),
                            cudaMemcpyHostToDevice, s);
            BatchDev b = B.dev();
            b.chunk_pre = B.tune_pre.p;
            launch_batch_flux(b, ph, plans[i], B.part.p, B.ldp, s);  // warm-up
            cudaEventRecord(ev0, s);
            for (int r = 0; r < 2; r++) launch_batch_flux(b, ph, plans[i], B.part.p, B.ldp, s);
            cudaEventRecord(ev1, s);
            if ((e = cudaEventSynchronize(ev1))) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            if (ms < best) {
                best = ms;
                pick = i;
            }
        }
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        if (e) return e;
        choice = PlanChoice{plans[pick].ppt, plans[pick].chunk};
        std::lock_guard<std::mutex> lk(g_plan_mu);
        g_plans.emplace(key, choice);  // a concurrent first measurement keeps its own
        choice = g_plans[key];
    }
    std::vector<int64_t> pre;
    B.plan = plan_for(B, choice.ppt, choice.chunk, pre);
    B.chunk_pre = pre;
    if ((e = B.part.ensure((size_t)std::max<int64_t>(B.plan.nchunk, 1) * (size_t)B.ldp)))
        return e;
    const size_t bytes = pre.size() * sizeof(int64_t);
    memcpy(B.tab<int64_t>(B.o_chunk), pre.data(), bytes);
    cudaMemcpyAsync(B.d_tab.p + B.o_chunk, B.h_tab + B.o_chunk, bytes, cudaMemcpyHostToDevice, s);
    return cudaSuccess;
}

// The stages of one batch on the context's stream.
// part: 0 every stage; 1 the table and the stages up to the phases; 2 the
// sweep, the reduction and the result copies (the first call of a layout
// runs 1, the flux autotuner, then 2).
void enqueue(lcg_ctx *c, BatchState &B, bool timed, int part = 0) {
    cudaStream_t s = c->stream;
    const BatchDev b = B.dev();
    const BatchPhases ph = B.phases();
    auto stage = [&](int id, auto &&fn) {
        Timer t;
        if (timed) c->stage_begin(id, t);
        fn();
        if (timed) c->stage_end(id, t);
    };
    if (part != 2) {
        cudaMemcpyAsync(B.d_tab.p, B.h_tab, B.tab_bytes, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(B.st.p, 0, (size_t)B.nmodels * sizeof(DevStatus), s);
        stage(LCG_STAGE_GRID, [&] { launch_batch_grid(b, c->nsm, s); });
        stage(LCG_STAGE_ECLIPSE, [&] { launch_batch_eclipse(b, c->nsm, c->eclipse_warp, s); });
        stage(LCG_STAGE_CONTINUUM, [&] { launch_batch_continuum(b, c->nsm, s); });
        stage(LCG_STAGE_FLATTEN, [&] { launch_batch_flatten(b, c->nsm, s); });
        stage(LCG_STAGE_PHASES, [&] { launch_batch_phases(b, c->data.p, c->off.p, B.n, ph, s); });
    }
    if (part == 1) return;
    stage(LCG_STAGE_FLUX, [&] { launch_batch_flux(b, ph, B.plan, B.part.p, B.ldp, s); });
    stage(LCG_STAGE_REDUCE, [&] {
        launch_batch_reduce(b, ph, B.part.p, B.ldp, B.osum.p, c->data.p, c->off.p, B.n,
                            B.flags & 3, B.calc.p, B.sfac.p, B.out.p, s);
    });
    const size_t nm = (size_t)B.nmodels;
    if (B.want_calc)
        cudaMemcpyAsync(B.h_res + B.r_calc, B.calc.p, nm * (size_t)B.n * 8,
                        cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(B.h_res + B.r_sfac, B.sfac.p, nm * 5 * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(B.h_res + B.r_out, B.out.p, nm * 3 * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(B.h_res + B.r_st, B.st.p, nm * sizeof(DevStatus), cudaMemcpyDeviceToHost,
                    s);
}

}  // namespace
}  // namespace eng
}  // namespace lcg

using namespace lcg;
using namespace lcg::eng;

extern "C" lcg_status lcg_light_curve_batch_resident(lcg_ctx *c, const lcg_model *models,
                                                     int32_t nmodels, int32_t flags,
                                                     double *sfac, double *calc, double *chisq,
                                                     double *wnok, int32_t *status) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    if (!models || nmodels < 0 || !sfac || !status) return c->fail(LCG_E_INVALID, "null argument");
    if (c->data_n < 1) return c->fail(LCG_E_INVALID, "no data: call lcg_set_data first");
    if (nmodels == 0) return LCG_OK;
    cudaSetDevice(c->device);
    const int32_t n = c->data_n;
    flags &= ~LCG_FLAG_DIAGNOSTICS;

    // which models go through the batch; the rest are evaluated one by one
    std::vector<uint8_t> inb((size_t)nmodels, 0);
    int32_t nb = 0;
    for (int32_t m = 0; m < nmodels; m++) {
        lcg_status rc = check_model(c, models + m);
        status[m] = rc;
        if (rc) continue;
        if (c->precision == LCG_PREC_MIXED && batchable(models[m])) {
            inb[m] = 1;
            nb++;
        }
    }
    c->err.clear();
    if (nb > 0) {
        if (!c->batch) c->batch = new BatchState();
        BatchState &B = *c->batch;
        const int want_calc = calc != nullptr;
        lcg_status rc;
        if (!same_layout(B, c, models, nmodels, flags, want_calc) &&
            (rc = relayout(c, B, models, nmodels, flags, want_calc))) {
            B.nmodels = -1;
            return rc;
        }
        // per-model host setup; geometry and continuum only where changed
        SlotDev *slots = B.tab<SlotDev>(B.o_slots);
        ModelDev *md = B.tab<ModelDev>(B.o_models);
        std::vector<uint8_t> geo((size_t)nmodels, 0), cont((size_t)nmodels, 0);
        std::vector<uint8_t> reuse((size_t)nmodels, 0);
        const double xmin = c->data_xmin, xmax = c->data_xmax;
        const bool same_data = B.data_version == c->data_version;
        // the same model as last time in its position, on the same points:
        // its previous results stand and nothing runs for it
        std::vector<int> todo;
        todo.reserve((size_t)nmodels);
        for (int32_t m = 0; m < nmodels; m++) {
            md[m].live = 0;
            slots[2 * m].live = slots[2 * m + 1].live = 0;
            if (!inb[m]) continue;
            if (same_data && B.key_ok[m] && memcmp(&B.key[m], models + m, sizeof(lcg_model)) == 0 &&
                ((flags & LCG_FLAG_SCALE) || B.key_sfac0[m] == sfac[5 * (size_t)m]))
                reuse[m] = 1;
            else
                todo.push_back(m);
        }
        parallel_for((int)todo.size(), [&](int j) {
            const int m = todo[(size_t)j];
            const lcg_model &M = models[m];
            ModelDev &D = md[m];
            SlotDev *S = slots + 2 * m;
            // light_curve_comp.cpp:130-154
            double r1, r2;
            get_r1r2(M, r1, r2);
            const double xl2 = xl12(M.q, M.spin2);
            if (xl2 < 0) {
                status[m] = LCG_E_NOCONVERGE;
                return;
            }
            if (r2 >= 0 && r2 > 1. - xl2) {
                status[m] = LCG_E_LOBE;
                return;
            }
            const bool g = !B.key_ok[m] || !same_geometry(B.key[m], M);
            const bool k = g || !same_continuum(B.key[m], M);
            if (g) {
                for (int star = 0; star < 2; star++) {
                    StarSetup su{};
                    Fail f{0, ""};
                    if (!prepare_star(M, star, 1, su, f, false)) {
                        status[m] = f.code;
                        return;
                    }
                    SlotDev &X = S[star];
                    const RingSet &R = B.slot_rings[2 * m + star];
                    GridParams &gp = X.gp;
                    gp.star = star;
                    gp.roche = star == kStar1 ? M.roche1 : M.roche2;
                    gp.npole = M.npole;
                    gp.nrings = R.nrings;
                    gp.nhalf = R.nhalf;
                    gp.q = M.q;
                    gp.spin = star == kStar1 ? M.spin1 : M.spin2;
                    gp.rref = star == kStar1 ? su.rref1 : su.rref2;
                    gp.pref = star == kStar1 ? su.pref1 : su.pref2;
                    gp.acc = M.delta_phase / 10.;
                    gp.gref = su.gref;
                    gp.rad_sphere = star == kStar1 ? su.r1 : su.r2;
                    EclParams &ep = X.ep;
                    ep.comp_star = star == kStar1 ? kStar2 : kStar1;
                    ep.comp_roche = star == kStar1 ? M.roche2 : M.roche1;
                    ep.q = M.q;
                    ep.comp_spin = star == kStar1 ? M.spin2 : M.spin1;
                    ep.comp_rref = star == kStar1 ? su.rref2 : su.rref1;
                    ep.comp_pref = star == kStar1 ? su.pref2 : su.pref1;
                    ep.comp_r = star == kStar1 ? su.r2 : su.r1;
                    const double ri = deg2rad(M.iangle);
                    ep.cosi = cos(ri);
                    ep.sini = sin(ri);
                    ep.delta = M.delta_phase;
                    set_ecl_screen(ep, 1, star == kStar1 ? su.r1 : su.r2);  // batches are mixed
                    X.eclipse_on = su.eclipse;
                }
            }
            if (k) {
                for (int star = 0; star < 2; star++) {
                    S[star].cp = continuum_params(M, star);
                    S[star].cp.fp32 = 1;  // batches are mixed
                    S[star].fc = fast_coef(M, star, 1);
                }
            }
            PhaseParams &pp = D.pp;
            pp.t0 = M.t0; pp.period = M.period; pp.pdot = M.pdot; pp.deltat = M.deltat;
            pp.slope = M.slope; pp.quad = M.quad; pp.cube = M.cube;
            pp.middle = (xmin + xmax) / 2.;
            pp.range = (xmax - xmin) / 2.;
            const double ri = deg2rad(M.iangle);
            pp.cosi = cos(ri);
            pp.sini = sin(ri);
            pp.gi = Ginterp{M.phase1, M.phase2, 1., 1., 1., 1.};
            D.third = M.third;
            D.sfac0 = sfac[5 * (size_t)m];
            D.live = 1;
            S[0].live = S[1].live = 1;
            geo[m] = g;
            cont[m] = k;
        });
        // work lists
        int32_t *counts = B.tab<int32_t>(B.o_counts);
        int32_t *gs = B.tab<int32_t>(B.o_geo_slot), *cs = B.tab<int32_t>(B.o_cont_slot);
        int64_t *gh = B.tab<int64_t>(B.o_geo_half), *gf = B.tab<int64_t>(B.o_geo_face);
        int64_t *cf = B.tab<int64_t>(B.o_cont_face), *cb = B.tab<int64_t>(B.o_cont_blk);
        int32_t ng = 0, nc = 0;
        gh[0] = gf[0] = cf[0] = cb[0] = 0;
        for (int32_t m = 0; m < nmodels; m++) {
            if (!md[m].live) continue;
            for (int star = 0; star < 2; star++) {
                const int s = 2 * m + star;
                const RingSet &R = B.slot_rings[s];
                if (geo[m]) {
                    gs[ng] = s;
                    gh[ng + 1] = gh[ng] + R.nhalf;
                    gf[ng + 1] = gf[ng] + R.nface;
                    ng++;
                }
                if (cont[m]) {
                    cs[nc] = s;
                    cf[nc + 1] = cf[nc] + R.nface;
                    cb[nc + 1] = cb[nc] + (R.nface + kSlotAlign - 1) / kSlotAlign;
                    nc++;
                }
            }
        }
        counts[0] = ng;
        counts[1] = nc;

        cudaError_t e;
        if (!B.tuned) {
            // first call on this layout: the stages up to the phases, the
            // measured flux plan, then the sweep with it
            enqueue(c, B, c->profiling, 1);
            if ((e = autotune_flux(c, B))) {
                cudaStreamSynchronize(c->stream);
                c->collect_timers();
                B.nmodels = -1;
                return c->cuda_fail(e, "flux autotuning");
            }
            B.tuned = true;
            enqueue(c, B, c->profiling, 2);
        } else if (c->profiling) {
            enqueue(c, B, true);
        } else {
            if (!B.exec) {
                cudaGraph_t graph = nullptr;
                if ((e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal)))
                    return c->cuda_fail(e, "batch capture");
                const int64_t k0 = lcg_kernel_launches(0);
                enqueue(c, B, false);
                B.graph_kernels = lcg_kernel_launches(0) - k0;
                count_launches(-B.graph_kernels);  // counted when the graph runs
                e = cudaStreamEndCapture(c->stream, &graph);
                if (e == cudaSuccess) e = cudaGraphInstantiate(&B.exec, graph, 0);
                if (graph) cudaGraphDestroy(graph);
                if (e) {
                    B.exec = nullptr;
                    return c->cuda_fail(e, "batch graph");
                }
            }
            if ((e = cudaGraphLaunch(B.exec, c->stream))) return c->cuda_fail(e, "batch launch");
            count_launches(B.graph_kernels);
        }
        if ((e = cudaStreamSynchronize(c->stream))) {
            c->collect_timers();
            B.nmodels = -1;  // relayout (and re-key every model) next time
            return c->cuda_fail(e, "batch");
        }
        c->collect_timers();
        const DevStatus *dst = B.res<DevStatus>(B.r_st);
        const double *hs = B.res<double>(B.r_sfac), *ho = B.res<double>(B.r_out);
        const double *hc = B.res<double>(B.r_calc);
        B.data_version = c->data_version;
        for (int32_t m = 0; m < nmodels; m++) {
            if (!inb[m]) continue;
            if (!reuse[m] && (!md[m].live || dst[m].code)) {
                if (!status[m]) status[m] = dst[m].code;
                B.key_ok[m] = 0;
                if (calc) memset(calc + (size_t)m * n, 0, (size_t)n * sizeof(double));
                continue;
            }
            if (!reuse[m]) {  // a reused model equals its key already
                B.key[m] = models[m];
                B.key_ok[m] = 1;
                B.key_sfac0[m] = sfac[5 * (size_t)m];
            }
            if (calc) memcpy(calc + (size_t)m * n, hc + (size_t)m * n, (size_t)n * sizeof(double));
            for (int k = 0; k < 5; k++) sfac[5 * (size_t)m + k] = hs[5 * (size_t)m + k];
            if (ho[3 * m + 2] != 0.) {
                if (chisq) chisq[m] = ho[3 * m];
                if (wnok) wnok[m] = ho[3 * m + 1];
            }
        }
        for (int32_t m = 0; m < nmodels; m++)
            if (md[m].live)
                c->flux_elements += (B.face0[2 * m + 2] - B.face0[2 * m]) * B.nent;
    }
    // the rest through the single-model path: on this context when there is
    // one, else concurrently on up to kWorkers worker contexts (same device,
    // precision and points; each model's arithmetic is that of the
    // single-model path, so the results are those of evaluating them one at
    // a time)
    std::vector<int32_t> rest;
    for (int32_t m = 0; m < nmodels; m++)
        if (!inb[m] && !status[m]) rest.push_back(m);
    auto one = [&](lcg_ctx *x, int32_t m) -> lcg_status {
        double sc[LCG_NOUT] = {0};
        if (chisq) sc[LCG_OUT_CHISQ] = chisq[m];
        if (wnok) sc[LCG_OUT_WNOK] = wnok[m];
        lcg_status rc = lcg_light_curve_resident(x, models + m, flags, sfac + 5 * (size_t)m,
                                                 calc ? calc + (size_t)m * n : nullptr, sc);
        status[m] = rc;
        if (rc) {
            if (calc) memset(calc + (size_t)m * n, 0, (size_t)n * sizeof(double));
            return rc;
        }
        if (chisq) chisq[m] = sc[LCG_OUT_CHISQ];
        if (wnok) wnok[m] = sc[LCG_OUT_WNOK];
        return LCG_OK;
    };
    constexpr int kWorkers = 8;
    const int nw = (int)std::min<size_t>(rest.size(), kWorkers);
    if (nw <= 1) {
        for (int32_t m : rest) {
            lcg_status rc = one(c, m);
            if (rc == LCG_E_CUDA || rc == LCG_E_NOMEM) return rc;
        }
        c->err.clear();
        return LCG_OK;
    }
    lcg_options o;
    lcg_default_options(&o);
    o.device = c->device;
    o.precision = c->precision;
    o.eclipse_warp = c->eclipse_warp;
    while ((int)c->workers.size() < nw) {
        lcg_ctx *w = nullptr;
        lcg_status rc = lcg_create(&w, &o);
        if (rc) return c->fail(rc, "creating a batch worker context");
        c->workers.push_back(w);
        c->worker_data_version.push_back(-1);
    }
    for (int k = 0; k < nw; k++)
        if (c->worker_data_version[k] != c->data_version) {
            lcg_status rc = lcg_set_data(c->workers[k],
                                         reinterpret_cast<const lcg_datum *>(c->h_data.data()),
                                         (int32_t)c->h_data.size());
            if (rc) return c->fail(rc, "resident points of a batch worker");
            c->worker_data_version[k] = c->data_version;
        }
    std::vector<lcg_status> fatal((size_t)nw, LCG_OK);
    std::vector<std::thread> threads;
    for (int k = 0; k < nw; k++)
        threads.emplace_back([&, k] {
            cudaSetDevice(c->device);
            for (size_t j = (size_t)k; j < rest.size(); j += (size_t)nw) {
                lcg_status rc = one(c->workers[k], rest[j]);
                if (rc == LCG_E_CUDA || rc == LCG_E_NOMEM) {
                    fatal[(size_t)k] = rc;
                    return;
                }
            }
        });
    for (auto &t : threads) t.join();
    for (lcg_status rc : fatal)
        if (rc) return rc;
    c->err.clear();
    return LCG_OK;
}

static lcg_status check_rows(lcg_ctx *c, const int32_t *rows, int32_t count, const void *out) {
    c->err.clear();
    if (!rows || !out || count < 0) return c->fail(LCG_E_INVALID, "null argument");
    BatchState *B = c->batch;
    if (!B || B->nmodels <= 0) return c->fail(LCG_E_INVALID, "no batch has run on this context");
    for (int32_t i = 0; i < count; i++)
        if (rows[i] < 0 || rows[i] >= B->nmodels)
            return c->fail(LCG_E_INVALID, "row %d outside the batch of %d", rows[i], B->nmodels);
    return LCG_OK;
}

extern "C" lcg_status lcg_batch_curves_device(lcg_ctx *c, const int32_t *rows, int32_t count,
                                              double *dst) {
    if (!c) return LCG_E_INVALID;
    cudaError_t e;
    if (!rows) {  // every row: one device copy of the curve matrix
        c->err.clear();
        BatchState *B = c->batch;
        if (!dst) return c->fail(LCG_E_INVALID, "null argument");
        if (!B || B->nmodels <= 0) return c->fail(LCG_E_INVALID, "no batch has run on this context");
        if (count != B->nmodels)
            return c->fail(LCG_E_INVALID, "count %d is not the batch's %d models", count, B->nmodels);
        cudaSetDevice(c->device);
        cudaMemcpyAsync(dst, B->calc.p, (size_t)count * B->n * sizeof(double),
                        cudaMemcpyDeviceToDevice, c->stream);
        if ((e = cudaStreamSynchronize(c->stream))) return c->cuda_fail(e, "curve rows");
        return LCG_OK;
    }
    lcg_status rc = check_rows(c, rows, count, dst);
    if (rc || count == 0) return rc;
    cudaSetDevice(c->device);
    BatchState *B = c->batch;
    if ((e = B->rows.ensure((size_t)count))) return c->cuda_fail(e, "curve rows");
    cudaMemcpyAsync(B->rows.p, rows, (size_t)count * sizeof(int32_t), cudaMemcpyHostToDevice,
                    c->stream);
    launch_gather_rows(B->calc.p, B->n, B->rows.p, count, dst, c->stream);
    if ((e = cudaStreamSynchronize(c->stream))) return c->cuda_fail(e, "curve rows");
    return LCG_OK;
}

extern "C" lcg_status lcg_batch_curves(lcg_ctx *c, const int32_t *rows, int32_t count,
                                       double *out) {
    if (!c) return LCG_E_INVALID;
    lcg_status rc = check_rows(c, rows, count, out);
    if (rc || count == 0) return rc;
    BatchState *B = c->batch;
    cudaSetDevice(c->device);
    const size_t n = (size_t)B->n, bytes = (size_t)count * n * sizeof(double);
    cudaError_t e;
    if ((e = B->rows.ensure((size_t)count)) || (e = B->gathered.ensure((size_t)count * n)))
        return c->cuda_fail(e, "curve rows");
    if (B->h_rows_cap < bytes) {
        if (B->h_rows) cudaFreeHost(B->h_rows);
        B->h_rows = nullptr;
        B->h_rows_cap = 0;
        if ((e = cudaHostAlloc((void **)&B->h_rows, bytes, cudaHostAllocDefault)))
            return c->cuda_fail(e, "curve rows");
        B->h_rows_cap = bytes;
    }
    cudaMemcpyAsync(B->rows.p, rows, (size_t)count * sizeof(int32_t), cudaMemcpyHostToDevice,
                    c->stream);
    launch_gather_rows(B->calc.p, B->n, B->rows.p, count, B->gathered.p, c->stream);
    cudaMemcpyAsync(B->h_rows, B->gathered.p, bytes, cudaMemcpyDeviceToHost, c->stream);
    if ((e = cudaStreamSynchronize(c->stream))) return c->cuda_fail(e, "curve rows");
    memcpy(out, B->h_rows, bytes);
    return LCG_OK;
}
