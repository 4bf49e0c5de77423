// The batching form behind hpm_run_batch: the runs of one pass over the views
// of a pyramid level share one launch per stage.
//
// The reference runs ProcessProblem for one view after another
// (main.cpp:1253-1255); each HPM::RunPatchMatch launches the initialisation and
// six half-sweeps over that view alone and synchronises after every launch
// (HPM.cu:2987-3035).  Here the runs' RunArgs go to device memory and each
// stage is one launch whose blocks are the tiles of all views (pm_kernels.cu,
// k_random_init_batch / k_half_sweep_batch), so the last wave of one view no
// longer idles the GPU.  Per-run setup (hypothesis reload, packing) and the
// hand-off of the results are the single-run code paths of run.cu, applied to
// per-run slices of resident batch buffers.
//
// Launch shapes of the half-sweep (block width 32, 16 or 8 pixels; one block
// per tile or a persistent grid; or, for views large enough to fill the GPU
// alone, one single-view launch per run, stage by stage) give the same
// results; the autotuner times them once per (source count, mode, size class)
// on a snapshot of the batch's state and restores the state before the real
// run.  With HPM_BATCH_GRAPH the
// initialisation and the half-sweeps are captured once per batch shape in a
// CUDA graph and replayed.
#include "ctx.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace hpm {

template <class T>
static cudaError_t ensure_dev(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

template <class T>
static cudaError_t ensure_pinned(T*& p, size_t& cap, size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost((void**)&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

static const int kBxCandidates[3] = { 32, 16, 8 };

// Sweep tiles of run k with blocks `bx` pixels wide: the per-view launch of
// pm_kernels.cu covers W x cover_pairs with blocks of bx x (block threads / bx).
static int sweep_tiles(const RunArgs& a, int bx, int block_threads) {
    const int rows = block_threads / bx;
    return ((a.W + bx - 1) / bx) * ((a.cover_pairs + rows - 1) / rows);
}

int Ctx::tune_batch(const BatchLaunch& base, int n, size_t total_px, uint64_t key, BatchShape& out) {
    // snapshot of everything a half-sweep writes; each candidate starts from it
    struct Buf { void* p; size_t bytes; };
    const Buf bufs[5] = { { b_planes, total_px * sizeof(float4) }, { b_costs, total_px * 4 },
                          { b_sel, total_px * 4 }, { b_rng, total_px * 4 }, { b_conf, total_px * 4 } };
    size_t snap_bytes = 0;
    for (const Buf& b : bufs) snap_bytes += b.bytes;
    uint8_t* snap = nullptr;
    cudaError_t e = cudaMalloc((void**)&snap, snap_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "autotuner snapshot");
    auto copy_all = [&](bool save) -> cudaError_t {
        size_t off = 0;
        for (const Buf& b : bufs) {
            cudaError_t r = save ? cudaMemcpyAsync(snap + off, b.p, b.bytes, cudaMemcpyDeviceToDevice, stream)
                                 : cudaMemcpyAsync(b.p, snap + off, b.bytes, cudaMemcpyDeviceToDevice, stream);
            if (r != cudaSuccess) return r;
            off += b.bytes;
        }
        return cudaSuccess;
    };
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int occ = half_sweep_batch_occupancy(base.max_s, base.mand);
    const int bt = half_sweep_block_threads(base.max_s);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int rc = HPM_OK;
    BatchShape best;
    best.ms = -1.0f;
    if ((e = cudaEventCreate(&t0)) != cudaSuccess || (e = cudaEventCreate(&t1)) != cudaSuccess) {
        rc = cuda_fail(e, "autotuner events");
    }
    if (!rc && (e = copy_all(true)) != cudaSuccess) rc = cuda_fail(e, "autotuner snapshot copy");
    for (int ci = 0; ci < 3 && !rc; ++ci) {
        const int bx = kBxCandidates[ci];
        if (bx > bt) continue;
        // tile table of this width, after the two tables of the run
        int* h = h_btiles + 2 * (n + 1);
        h[0] = 0;
        for (int k = 0; k < n; ++k) h[k + 1] = h[k] + sweep_tiles(h_bargs[k], bx, bt);
        int* d = d_btiles + 2 * (n + 1);
        if ((e = cudaMemcpyAsync(d, h, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
            rc = cuda_fail(e, "autotuner tiles");
            break;
        }
        for (int persist = 0; persist <= 2 && !rc; ++persist) {
            BatchLaunch bl = base;
            bl.count = false;
            bl.tile_start = d;
            bl.tiles = h[n];
            bl.bx = bx;
            bl.grid_blocks = persist ? persist * occ * sms : 0;
            if (persist && bl.grid_blocks >= bl.tiles) continue;
            if ((e = copy_all(false)) != cudaSuccess) { rc = cuda_fail(e, "autotuner restore"); break; }
            cudaEventRecord(t0, stream);
            if ((e = launch_half_sweep_batch(bl, 0, 0, stream)) != cudaSuccess) { rc = cuda_fail(e, "autotuner launch"); break; }
            cudaEventRecord(t1, stream);
            ++launches;
            if ((e = cudaEventSynchronize(t1)) != cudaSuccess) { rc = cuda_fail(e, "autotuner timing"); break; }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, t0, t1);
            if (best.ms < 0.0f || ms < best.ms) {
                best.ms = ms;
                best.bx = bx;
                best.persist = persist;
            }
        }
    }
    // the single-view kernel, one launch per run: its RunArgs are kernel parameters, not device memory
    if (!rc && (e = copy_all(false)) != cudaSuccess) rc = cuda_fail(e, "autotuner restore");
    if (!rc) {
        cudaEventRecord(t0, stream);
        for (int k = 0; k < n && !rc; ++k) {
            if ((e = launch_half_sweep(h_bargs[k], 0, 0, stream)) != cudaSuccess) rc = cuda_fail(e, "autotuner launch");
            ++launches;
        }
        cudaEventRecord(t1, stream);
        if (!rc && (e = cudaEventSynchronize(t1)) != cudaSuccess) rc = cuda_fail(e, "autotuner timing");
        float ms = 0.0f;
        if (!rc) cudaEventElapsedTime(&ms, t0, t1);
        if (!rc && (best.ms < 0.0f || ms < best.ms)) {
            best.ms = ms;
            best.bx = 32;
            best.persist = 0;
            best.perview = true;
        }
    }
    if (!rc && (e = copy_all(false)) != cudaSuccess) rc = cuda_fail(e, "autotuner restore");
    if (!rc && (e = cudaStreamSynchronize(stream)) != cudaSuccess) rc = cuda_fail(e, "autotuner");
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(snap);
    if (rc) return rc;
    out = best;
    batch_shapes.emplace_back(key, best);
    return HPM_OK;
}

int Ctx::run_batch(int n, const int32_t* refs, const int32_t* src_off, const int32_t* src_ids,
                   const hpm_params* params, int texture_level, const uint64_t* seeds) {
    cudaSetDevice(device);
    if (n < 1 || n > HPM_MAX_VIEWS || !refs || !src_off || !src_ids || !params || !seeds)
        return fail(HPM_E_INVALID, "hpm_run_batch: bad arguments");
    const uint32_t mode = params[0].mode & ~(uint32_t)HPM_MODE_UPSAMPLE;
    const int iters = params[0].max_iterations;
    if (iters < 0 || iters > 32) return fail(HPM_E_INVALID, "hpm_run_batch: max_iterations must be 0..32");
    const bool geom = mode & HPM_MODE_GEOM, prior = mode & HPM_MODE_PRIOR, hier = mode & HPM_MODE_HIERARCHY;
    const bool mand = mode & HPM_MODE_MAND;
    std::vector<char> seen(HPM_MAX_VIEWS, 0);
    size_t total = 0, total_scaled = 0;
    int max_s = 0;
    for (int k = 0; k < n; ++k) {
        const int r = refs[k];
        if (r < 0 || r >= HPM_MAX_VIEWS || views[r].w == 0) return fail(HPM_E_STATE, "reference view %d not set", r);
        if (seen[r]) return fail(HPM_E_INVALID, "hpm_run_batch: view %d appears twice", r);
        seen[r] = 1;
        if ((params[k].mode & ~(uint32_t)HPM_MODE_UPSAMPLE) != mode)
            return fail(HPM_E_INVALID, "hpm_run_batch: the runs of a batch share one mode");
        if (params[k].max_iterations != iters)
            return fail(HPM_E_INVALID, "hpm_run_batch: the runs of a batch share one iteration count");
        const int ns = src_off[k + 1] - src_off[k];
        if (ns < 1 || ns > HPM_MAX_SRC) return fail(HPM_E_INVALID, "hpm_run_batch: run %d has %d sources (1..31)", k, ns);
        max_s = std::max(max_s, ns);
        total += (size_t)views[r].w * views[r].h;
        if (hier && !geom && !prior) {
            const DevMap& nm = views[r].maps[HPM_MAP_NORMAL];
            if (!nm.ptr) return fail(HPM_E_STATE, "hierarchy: view %d lacks coarse normal/cost maps", r);
            total_scaled += (size_t)nm.w * nm.h;
        }
    }
    cudaError_t e;
    if ((e = ensure_dev(b_planes, b_cap_planes, total)) != cudaSuccess ||
        (e = ensure_dev(b_costs, b_cap_costs, total)) != cudaSuccess ||
        (e = ensure_dev(b_pre, b_cap_pre, total)) != cudaSuccess ||
        (e = ensure_dev(b_sel, b_cap_sel, total)) != cudaSuccess ||
        (e = ensure_dev(b_rng, b_cap_rng, total)) != cudaSuccess ||
        (e = ensure_dev(b_conf, b_cap_conf, total)) != cudaSuccess ||
        (e = ensure_dev(b_scaled, b_cap_scaled, total_scaled)) != cudaSuccess ||
        (e = ensure_dev(d_bargs, d_bargs_cap, (size_t)n)) != cudaSuccess ||
        (e = ensure_dev(d_btiles, d_btiles_cap, (size_t)3 * (n + 1))) != cudaSuccess ||
        (e = ensure_pinned(h_bargs, h_bargs_cap, (size_t)n)) != cudaSuccess ||
        (e = ensure_pinned(h_btiles, h_btiles_cap, (size_t)3 * (n + 1))) != cudaSuccess)
        return cuda_fail(e, "alloc batch buffers");
    // the staging of the previous batch may still be read by its copies
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "hpm_run_batch");

    size_t off = 0, soff = 0;
    for (int k = 0; k < n; ++k) {
        const int r = refs[k];
        RunBufs b;
        b.planes = b_planes + off; b.costs = b_costs + off; b.pre_costs = b_pre + off;
        b.sel = b_sel + off; b.rng = b_rng + off; b.conf = b_conf + off;
        if (hier && !geom && !prior) {
            b.scaled = b_scaled + soff;
            soff += (size_t)views[r].maps[HPM_MAP_NORMAL].w * views[r].maps[HPM_MAP_NORMAL].h;
        }
        const int ns = src_off[k + 1] - src_off[k];
        int rc = prepare_run_into(r, src_ids + src_off[k], ns, &params[k], texture_level, seeds[k], b, h_bargs[k]);
        if (rc) return rc;
        off += (size_t)views[r].w * views[r].h;
    }

    // prior mode: work lists of every run (confidences and prior masks are fixed during the pass and the
    // initialisation does not change them), computed before the launches that a graph may replay
    const bool listed = prior && !mand && iters > 0;
    if (listed) {
        size_t words = 0;
        for (int k = 0; k < n; ++k) words += 2 * (size_t)h_bargs[k].cover_pairs * (h_bargs[k].W + 1);
        if ((e = ensure_dev(b_active, b_active_cap, words)) != cudaSuccess) return cuda_fail(e, "alloc prior work lists");
        size_t w = 0;
        for (int k = 0; k < n; ++k) {
            RunArgs& a = h_bargs[k];
            int* px = b_active + w;
            int* cnt = px + 2 * (size_t)a.cover_pairs * a.W;
            w += 2 * (size_t)a.cover_pairs * (a.W + 1);
            if ((e = launch_prior_active(a, px, cnt, stream)) != cudaSuccess) return cuda_fail(e, "prior work lists");
            ++launches;
            a.active_px = px;
            a.active_n = cnt;
        }
    }

    // tile tables: initialisation (16 x 8 pixel blocks), then the half-sweep's
    const int bt = half_sweep_block_threads(max_s);
    const uint64_t key = (uint64_t)max_s | ((uint64_t)mand << 8) |
                         ((uint64_t)(total ? (int)std::log2((double)total) : 0) << 16);
    BatchShape shape;
    bool have_shape = false;
    if (batch_flags & HPM_BATCH_PER_VIEW) {
        shape.perview = true;
        have_shape = true;
    } else {
        for (const auto& kv : batch_shapes)
            if (kv.first == key) { shape = kv.second; have_shape = true; }
    }
    int* hi = h_btiles;
    hi[0] = 0;
    for (int k = 0; k < n; ++k) hi[k + 1] = hi[k] + ((h_bargs[k].W + 15) / 16) * ((h_bargs[k].H + 7) / 8);
    auto fill_sweep = [&](int bx) {
        int* hs = h_btiles + (n + 1);
        hs[0] = 0;
        for (int k = 0; k < n; ++k) hs[k + 1] = hs[k] + sweep_tiles(h_bargs[k], bx, bt);
    };
    fill_sweep(shape.bx);
    if ((e = cudaMemcpyAsync(d_bargs, h_bargs, sizeof(RunArgs) * n, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_btiles, h_btiles, sizeof(int) * 2 * (n + 1), cudaMemcpyHostToDevice, stream)) !=
            cudaSuccess)
        return cuda_fail(e, "upload batch");

    BatchLaunch bi{};
    bi.args = d_bargs;
    bi.tile_start = d_btiles;
    bi.n = n;
    bi.tiles = hi[n];
    bi.max_s = max_s;
    bi.grid_blocks = 0;
    bi.mand = mand;
    bi.listed = listed;
    bi.count = (prof_flags & HPM_PROFILE_COUNT) && prof_hyp;
    BatchLaunch bs = bi;
    bs.tile_start = d_btiles + (n + 1);
    bs.tiles = h_btiles[(n + 1) + n];
    bs.bx = shape.bx;

    // one half-sweep stage of every run: one batched launch, or the single-view kernel per run
    auto sweep_stage = [&](int color, int iter, TimedLaunch*& t) -> int {
        int r = HPM_OK;
        if (!shape.perview) {
            if ((r = record_start(1, t))) return r;
            if ((e = launch_half_sweep_batch(bs, color, iter, stream)) != cudaSuccess)
                return cuda_fail(e, "batched half sweep");
            if (t) cudaEventRecord(t->stop, stream);
            ++launches;
            return HPM_OK;
        }
        for (int k = 0; k < n; ++k) {
            if ((r = record_start(1, t))) return r;
            if ((e = launch_half_sweep(h_bargs[k], color, iter, stream)) != cudaSuccess)
                return cuda_fail(e, "half sweep");
            if (t) cudaEventRecord(t->stop, stream);
            ++launches;
        }
        return HPM_OK;
    };
    const bool timing = prof_flags & HPM_PROFILE_TIMING;
    const bool use_graph = (batch_flags & HPM_BATCH_GRAPH) && !timing && !bi.count;
    TimedLaunch* t = nullptr;
    int rc = HPM_OK;
    // the schedule: initialisation, then 2 x iters half-sweeps (RunPatchMatch, HPM.cu:3013-3021)
    auto schedule = [&]() -> int {
        if ((rc = record_start(0, t))) return rc;
        if ((e = launch_random_init_batch(bi, stream)) != cudaSuccess) return cuda_fail(e, "batched init launch");
        if (t) cudaEventRecord(t->stop, stream);
        ++launches;
        for (int k = 0; k < 2 * iters; ++k)
            if ((rc = sweep_stage(k & 1, k >> 1, t))) return rc;
        return HPM_OK;
    };
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    auto set_grid = [&]() {
        bs.grid_blocks = shape.persist ? shape.persist * half_sweep_batch_occupancy(max_s, mand) * sms : 0;
    };
    set_grid();
    // a graph of per-view launches would hold this batch's RunArgs as parameters; the batched kernels read
    // theirs from device memory, refreshed before every replay
    BatchGraph* graph = nullptr;
    if (use_graph && have_shape && !shape.perview)
        for (auto& g : batch_graphs)
            if (g.n == n && g.init_tiles == bi.tiles && g.sweep_tiles == bs.tiles && g.max_s == max_s &&
                g.mand == mand && g.iters == iters && g.bx == bs.bx && g.grid == bs.grid_blocks &&
                g.perview == shape.perview)
                graph = &g;
    if (graph) {
        if ((e = cudaGraphLaunch(graph->exec, stream)) != cudaSuccess) return cuda_fail(e, "batch graph launch");
        launches += 1 + 2 * iters * (shape.perview ? n : 1);
    } else if (!have_shape && (batch_flags & HPM_BATCH_AUTOTUNE) && iters > 0) {
        // initialise, tune the half-sweep on a snapshot of the initialised state, then sweep
        if ((rc = record_start(0, t))) return rc;
        if ((e = launch_random_init_batch(bi, stream)) != cudaSuccess) return cuda_fail(e, "batched init launch");
        if (t) cudaEventRecord(t->stop, stream);
        ++launches;
        if ((rc = tune_batch(bs, n, total, key, shape))) return rc;
        fill_sweep(shape.bx);
        if ((e = cudaMemcpyAsync(d_btiles + (n + 1), h_btiles + (n + 1), sizeof(int) * (n + 1),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_fail(e, "upload batch tiles");
        bs.tiles = h_btiles[(n + 1) + n];
        bs.bx = shape.bx;
        set_grid();
        for (int k = 0; k < 2 * iters; ++k)
            if ((rc = sweep_stage(k & 1, k >> 1, t))) return rc;
    } else {
        if ((rc = schedule())) return rc;
        if (use_graph && !shape.perview) {
            // record the same launches (not executed) for the next batch of this shape
            cudaGraph_t g = nullptr;
            if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed)) != cudaSuccess)
                return cuda_fail(e, "batch graph capture");
            const int64_t l0 = launches;
            const int crc = schedule();
            const cudaError_t ce = cudaStreamEndCapture(stream, &g);
            launches = l0;
            if (crc) { if (g) cudaGraphDestroy(g); return crc; }
            if (ce != cudaSuccess) return cuda_fail(ce, "batch graph capture");
            cudaGraphExec_t ex = nullptr;
            e = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
            BatchGraph bg;
            bg.n = n; bg.init_tiles = bi.tiles; bg.sweep_tiles = bs.tiles; bg.max_s = max_s; bg.mand = mand;
            bg.iters = iters; bg.bx = bs.bx; bg.grid = bs.grid_blocks; bg.perview = shape.perview; bg.exec = ex;
            batch_graphs.push_back(bg);
        }
    }
    for (int k = 0; k < n; ++k) {
        rc = finish_run(refs[k], h_bargs[k], geom);
        if (rc) return rc;
    }
    return HPM_OK;
}

}  // namespace hpm
