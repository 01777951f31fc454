// Continuous-batching request server (no reference counterpart: the reference only offers blocking
// batch calls).  It replays an open-loop request trace in real time:
//   * requests (sign or verify, parameter set 2/3/5, key index, message) become visible at their
//     arrival time and wait in one FIFO per (parameter set, operation) lane;
//   * every lane owns several batch slots (a stream, device buffers and, for the fused path, an
//     engine sharing the parameter set's resident key caches); a free slot immediately takes
//     everything its lane has queued (up to max_batch) and runs it on the GPU while newly arriving
//     requests queue for the next free slot, so batches of one lane and of different lanes overlap
//     on the device;
//   * slots are created only as far as the device-memory budget allows (admission by budget):
//     requests wait on the host until a slot, and with it its memory, is free again.
// The same loop runs the plain stage-by-stage path (no key caches: key material is expanded per
// batch) for comparison.  Latency = completion time observed on the host - arrival time.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cudilithium.h"

namespace cudil {
int cudil_record_cuda_error(cudaError_t e, const char *file, int line);
}
#define SRV_CK(x)                                                                              \
    do {                                                                                       \
        const cudaError_t srv_e_ = (x);                                                        \
        if (srv_e_ != cudaSuccess) return ::cudil::cudil_record_cuda_error(srv_e_, __FILE__, __LINE__); \
    } while (0)

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kModes[3] = {2, 3, 5};
inline int mode_index(int mode) { return mode == 2 ? 0 : (mode == 3 ? 1 : (mode == 5 ? 2 : -1)); }
inline size_t al8(size_t x) { return (x + 7) / 8 * 8; }

struct Trace {
    const cudil_request *reqs;
    size_t n;
    const uint8_t *msgs;
    const uint8_t *sigs;
    const uint8_t *sk[3];
    const uint8_t *pk[3];
    size_t nkeys[3];
    cudil_params prm[3];
    uint8_t *sig_out;
    size_t sig_out_pitch;
    cudil_request_result *res;
    Clock::time_point t0;
};

struct Slot {
    int lane = 0, mode = 0, op = 0;
    const cudil_serve_config *cfg = nullptr;
    Trace *tr = nullptr;
    cudaStream_t st = nullptr;
    // fused
    cudil_engine *eng = nullptr;
    // plain
    uint8_t *pool = nullptr, *tpool = nullptr;
    size_t pitch = 0, tpitch = 0;
    cudil_task_lut lut{};
    std::vector<cudil_sign_lut_element> sign_lut;
    uint32_t *d_mlens = nullptr;
    uint8_t *d_keys = nullptr;
    // shared
    uint8_t *d_msgs = nullptr, *d_sig = nullptr;
    int *d_ret = nullptr;
    uint8_t *h_msgs = nullptr, *h_sig = nullptr, *h_keys = nullptr;
    int *h_ret = nullptr;
    uint32_t *h_mlens = nullptr;
    size_t msgs_cap = 0, max_batch = 0;
    std::vector<unsigned long long> off;
    std::vector<uint32_t> mlen, key;
    // work hand-off
    std::mutex mu;
    std::condition_variable cv;
    std::vector<uint32_t> batch;
    bool has_work = false, stop = false;
    std::atomic<bool> busy{false};
    std::atomic<int> error{0};
    std::thread worker;
    std::atomic<size_t> *completed = nullptr;
    std::atomic<size_t> batches{0}, items{0};
    // host-side time split of this slot's batches (ns): staging into pinned buffers, from the
    // first copy/launch to the stream's completion, result write-back
    std::atomic<unsigned long long> stage_ns{0}, device_ns{0}, post_ns{0};

    size_t device_bytes = 0;

    // record = false: a warm-up batch (graph capture, first-touch of buffers) whose results are
    // dropped.
    int run_batch(bool record = true) {
        const cudil_params &p = tr->prm[mode_index(mode)];
        const size_t n = batch.size();
        const size_t sigb = p.sig_bytes;
        const auto c0 = Clock::now();
        // stage messages (fused: packed at 8-byte aligned offsets; plain: rows of cfg->max_mlen)
        size_t pos = 0;
        for (size_t i = 0; i < n; ++i) {
            const cudil_request &r = tr->reqs[batch[i]];
            if (cfg->path == 0) {
                off[i] = pos;
                std::memcpy(h_msgs + pos, tr->msgs + r.msg_off, r.mlen);
                pos += al8(r.mlen);
            } else {
                std::memcpy(h_msgs + i * cfg->max_mlen, tr->msgs + r.msg_off, r.mlen);
                h_mlens[i] = r.mlen;
            }
            mlen[i] = r.mlen;
            key[i] = r.key;
            if (op == 1) std::memcpy(h_sig + i * sigb, tr->sigs + r.sig_off, sigb);
        }
        const size_t msg_bytes = (cfg->path == 0) ? std::max<size_t>(pos, 8) : n * cfg->max_mlen;
        const auto c1 = Clock::now();
        SRV_CK(cudaMemcpyAsync(d_msgs, h_msgs, msg_bytes, cudaMemcpyHostToDevice, st));
        if (op == 1) SRV_CK(cudaMemcpyAsync(d_sig, h_sig, n * sigb, cudaMemcpyHostToDevice, st));
        int rc = CUDIL_OK;
        const int mi = mode_index(mode);
        if (cfg->path == 0) {
            if (op == 0)
                rc = cudil_engine_sign(eng, d_sig, d_msgs, msg_bytes, off.data(), mlen.data(), key.data(), n, st);
            else
                rc = cudil_engine_verify(eng, d_ret, d_sig, d_msgs, msg_bytes, off.data(), mlen.data(), key.data(), n, st);
        } else {
            // plain path: per-item key material gathered into rows, key expansion inside the call
            const size_t kb = (op == 0) ? (size_t)p.sk_bytes : (size_t)p.pk_bytes;
            const uint8_t *src = (op == 0) ? tr->sk[mi] : tr->pk[mi];
            for (size_t i = 0; i < n; ++i) std::memcpy(h_keys + i * kb, src + (size_t)key[i] * kb, kb);
            if (cudaMemcpyAsync(d_keys, h_keys, n * kb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(d_mlens, h_mlens, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
                return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
            if (op == 0) {
                sign_lut.assign(n, cudil_sign_lut_element{0, 0});
                lut.sign_lut = sign_lut.data();
                lut.sign_lut_len = n;
                rc = cudil_sign_dev_varlen(mode, d_sig, sigb, d_msgs, cfg->max_mlen, d_mlens, cfg->max_mlen, d_keys, pool,
                                           pitch, tpool, tpitch, &lut, (size_t)cfg->plain_exec_threshold, n, st);
            } else {
                rc = cudil_verify_dev_varlen(mode, d_ret, d_sig, sigb, sigb, d_msgs, cfg->max_mlen, d_mlens, cfg->max_mlen,
                                             d_keys, pool, pitch, n, st);
            }
        }
        if (rc) return rc;
        if (op == 0) {
            SRV_CK(cudaMemcpyAsync(h_sig, d_sig, n * sigb, cudaMemcpyDeviceToHost, st));
        } else {
            SRV_CK(cudaMemcpyAsync(h_ret, d_ret, n * sizeof(int), cudaMemcpyDeviceToHost, st));
        }
        SRV_CK(cudaStreamSynchronize(st));
        const auto c2 = Clock::now();
        if (cfg->path == 0 && op == 0) {
            unsigned long long att = 0;
            unsigned err = 0;
            if (cudil_engine_last_status(eng, &att, &err) != CUDIL_OK) return CUDIL_ERR_TIMEOUT;
        }
        if (!record) return CUDIL_OK;
        const double done = std::chrono::duration<double>(Clock::now() - tr->t0).count();
        for (size_t i = 0; i < n; ++i) {
            const uint32_t ri = batch[i];
            tr->res[ri].done_s = done;
            tr->res[ri].status = (op == 0) ? 0 : h_ret[i];
            tr->res[ri].batch_size = (uint32_t)n;
            if (op == 0 && tr->sig_out) std::memcpy(tr->sig_out + (size_t)ri * tr->sig_out_pitch, h_sig + i * sigb, sigb);
        }
        batches += 1;
        items += n;
        auto ns = [](Clock::duration d) { return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(d).count(); };
        stage_ns += ns(c1 - c0);
        device_ns += ns(c2 - c1);
        post_ns += ns(Clock::now() - c2);
        return CUDIL_OK;
    }

    void loop(int device) {
        cudaSetDevice(device);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return has_work || stop; });
                if (stop && !has_work) return;
            }
            const int rc = run_batch();
            if (rc) error = rc;
            const size_t n = batch.size();
            completed->fetch_add(n);
            {
                // busy is cleared under the same lock that published the work, after the batch is
                // consumed, so the dispatcher never sees a free slot that still holds a batch
                std::lock_guard<std::mutex> lk(mu);
                has_work = false;
                batch.clear();
                busy = false;
            }
        }
    }

    void release() {
        if (st) cudaStreamDestroy(st);
        if (eng) cudil_engine_destroy(eng);
        cudaFree(pool);
        cudaFree(tpool);
        cudaFree(d_mlens);
        cudaFree(d_keys);
        cudaFree(d_msgs);
        cudaFree(d_sig);
        cudaFree(d_ret);
        cudaFree(lut.d_exec_lut);
        cudaFree(lut.d_done_lut);
        cudaFree(lut.d_copy_lut);
        if (lut.h_exec_lut) cudaFreeHost(lut.h_exec_lut);
        if (lut.h_done_lut) cudaFreeHost(lut.h_done_lut);
        if (lut.h_copy_lut) cudaFreeHost(lut.h_copy_lut);
        if (h_msgs) cudaFreeHost(h_msgs);
        if (h_sig) cudaFreeHost(h_sig);
        if (h_keys) cudaFreeHost(h_keys);
        if (h_ret) cudaFreeHost(h_ret);
        if (h_mlens) cudaFreeHost(h_mlens);
    }
};

inline size_t pitch512(size_t x) { return (x + 511) / 512 * 512; }

// Device bytes of a slot's own buffers (the fused engine's are added by the engine itself).
size_t slot_buffer_bytes(const cudil_serve_config *cfg, const cudil_params &p, int op) {
    const size_t B = (size_t)cfg->max_batch;
    const size_t msgs_cap = (cfg->path == 0) ? B * al8(cfg->max_mlen) + 8 : B * (size_t)cfg->max_mlen + 8;
    size_t b = msgs_cap + B * p.sig_bytes + B * sizeof(int);
    if (cfg->path == 1) {
        const size_t T = (size_t)cfg->plain_exec_threshold;
        b += B * ((op == 0 ? (size_t)p.sk_bytes : (size_t)p.pk_bytes) + sizeof(uint32_t));
        if (op == 0)
            b += B * pitch512(cudil_sign_row_bytes(p.mode, cfg->max_mlen)) + T * pitch512(cudil_sign_temp_row_bytes(p.mode)) +
                 T * (4 + 1 + sizeof(cudil_copy_lut_element));
        else
            b += B * pitch512(cudil_verify_row_bytes(p.mode, cfg->max_mlen));
    }
    return b;
}

// Creates one slot of a lane inside `remaining` device bytes (0 = unlimited).  CUDIL_ERR_BUDGET:
// the slot does not fit and nothing stays allocated.
int make_slot(Slot &s, const cudil_serve_config *cfg, Trace *tr, cudil_engine *const *cache, size_t remaining) {
    const int mi = mode_index(s.mode);
    const cudil_params &p = tr->prm[mi];
    const size_t B = (size_t)cfg->max_batch;
    const size_t own = slot_buffer_bytes(cfg, p, s.op);
    if (remaining && own >= remaining) return CUDIL_ERR_BUDGET;
    s.max_batch = B;
    s.cfg = cfg;
    s.tr = tr;
    s.off.resize(B);
    s.mlen.resize(B);
    s.key.resize(B);
    if (cfg->path == 0) {
        // the engine checks its own requirement against what is left before allocating
        int rc = cudil_engine_create(&s.eng, s.mode, 0, B, cfg->engine_threads, remaining ? remaining - own : 0);
        if (rc) return rc;
        rc = cudil_engine_attach_keys(s.eng, cache[mi]);
        if (rc) return rc;
        if (cfg->engine_spec_slots) cudil_engine_set_spec_slots(s.eng, (unsigned)cfg->engine_spec_slots);
    }
    SRV_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    s.msgs_cap = (cfg->path == 0) ? B * al8(cfg->max_mlen) + 8 : B * (size_t)cfg->max_mlen + 8;
    if (cudaMalloc(&s.d_msgs, s.msgs_cap) != cudaSuccess || cudaMalloc(&s.d_sig, B * p.sig_bytes) != cudaSuccess ||
        cudaMalloc(&s.d_ret, B * sizeof(int)) != cudaSuccess || cudaMallocHost(&s.h_msgs, s.msgs_cap) != cudaSuccess ||
        cudaMallocHost(&s.h_sig, B * p.sig_bytes) != cudaSuccess || cudaMallocHost(&s.h_ret, B * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&s.h_mlens, B * sizeof(uint32_t)) != cudaSuccess)
        return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
    if (cfg->path == 1) {
        const size_t kb = (s.op == 0) ? (size_t)p.sk_bytes : (size_t)p.pk_bytes;
        if (cudaMalloc(&s.d_keys, B * kb) != cudaSuccess || cudaMalloc(&s.d_mlens, B * sizeof(uint32_t)) != cudaSuccess ||
            cudaMallocHost(&s.h_keys, B * kb) != cudaSuccess)
            return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        if (s.op == 0) {
            const size_t T = (size_t)cfg->plain_exec_threshold;
            s.pitch = pitch512(cudil_sign_row_bytes(s.mode, cfg->max_mlen));
            s.tpitch = pitch512(cudil_sign_temp_row_bytes(s.mode));
            if (cudaMalloc(&s.pool, B * s.pitch) != cudaSuccess || cudaMalloc(&s.tpool, T * s.tpitch) != cudaSuccess ||
                cudaMalloc(&s.lut.d_exec_lut, T * 4) != cudaSuccess || cudaMalloc(&s.lut.d_done_lut, T) != cudaSuccess ||
                cudaMalloc(&s.lut.d_copy_lut, T * sizeof(cudil_copy_lut_element)) != cudaSuccess ||
                cudaMallocHost(&s.lut.h_exec_lut, T * 4) != cudaSuccess || cudaMallocHost(&s.lut.h_done_lut, T) != cudaSuccess ||
                cudaMallocHost(&s.lut.h_copy_lut, T * sizeof(cudil_copy_lut_element)) != cudaSuccess)
                return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        } else {
            s.pitch = pitch512(cudil_verify_row_bytes(s.mode, cfg->max_mlen));
            SRV_CK(cudaMalloc(&s.pool, B * s.pitch));
        }
    }
    s.device_bytes = own + (s.eng ? cudil_engine_device_bytes(s.eng) : 0);
    return CUDIL_OK;
}

}  // namespace

extern "C" int cudil_serve_trace(const cudil_serve_config *cfg, const uint8_t *const sk[3], const uint8_t *const pk[3],
                                 const size_t nkeys[3], const cudil_request *reqs, size_t nreq, const uint8_t *msgs,
                                 const uint8_t *sigs, uint8_t *sig_out, size_t sig_out_pitch,
                                 cudil_request_result *results, cudil_serve_stats *stats) {
    if (!cfg || !reqs || !results || cfg->max_batch <= 0 || cfg->slots_per_lane <= 0 || cfg->max_mlen == 0 ||
        (cfg->path != 0 && cfg->path != 1) || (cfg->path == 1 && cfg->plain_exec_threshold <= 0))
        return CUDIL_ERR_INVALID;
    Trace tr{};
    tr.reqs = reqs;
    tr.n = nreq;
    tr.msgs = msgs;
    tr.sigs = sigs;
    tr.sig_out = sig_out;
    tr.sig_out_pitch = sig_out_pitch;
    tr.res = results;
    bool used[3] = {false, false, false};
    for (int m = 0; m < 3; ++m) {
        tr.sk[m] = sk ? sk[m] : nullptr;
        tr.pk[m] = pk ? pk[m] : nullptr;
        tr.nkeys[m] = nkeys ? nkeys[m] : 0;
        cudil_get_params(kModes[m], &tr.prm[m]);
    }
    for (size_t i = 0; i < nreq; ++i) {
        const cudil_request &r = reqs[i];
        const int mi = mode_index(r.mode);
        if (mi < 0 || (r.op != 0 && r.op != 1) || r.key >= tr.nkeys[mi] || r.mlen > cfg->max_mlen ||
            (r.op == 0 && !tr.sk[mi]) || (r.op == 1 && (!tr.pk[mi] || !sigs)))
            return CUDIL_ERR_INVALID;
        if (i && r.arrival_s < reqs[i - 1].arrival_s) return CUDIL_ERR_INVALID;  // trace must be in arrival order
        used[mi] = true;
    }
    int device = 0;
    SRV_CK(cudaGetDevice(&device));

    // resident key caches (fused path): one cache engine per parameter set
    cudil_engine *cache[3] = {nullptr, nullptr, nullptr};
    size_t used_bytes = 0;
    int rc = CUDIL_OK;
    std::vector<std::unique_ptr<Slot>> slots;
    auto cleanup = [&]() {
        for (auto &s : slots) {
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->stop = true;
            }
            s->cv.notify_all();
            if (s->worker.joinable()) s->worker.join();
            s->release();
        }
        for (auto &c : cache)
            if (c) cudil_engine_destroy(c);
    };
    if (cfg->path == 0) {
        for (int m = 0; m < 3 && rc == CUDIL_OK; ++m) {
            if (!used[m]) continue;
            const cudil_params &p = tr.prm[m];
            rc = cudil_engine_create(&cache[m], kModes[m], tr.nkeys[m], 0, cfg->engine_threads,
                                     cfg->device_budget_bytes ? (used_bytes < cfg->device_budget_bytes
                                                                     ? cfg->device_budget_bytes - used_bytes
                                                                     : 1)
                                                              : 0);
            if (rc) break;
            uint8_t *d = nullptr;
            const size_t kbytes = tr.nkeys[m] * (size_t)std::max(p.sk_bytes, p.pk_bytes);
            if (cudaMalloc(&d, kbytes) != cudaSuccess) {
                rc = ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
                break;
            }
            if (tr.sk[m]) {
                cudaMemcpy(d, tr.sk[m], tr.nkeys[m] * p.sk_bytes, cudaMemcpyHostToDevice);
                rc = cudil_engine_set_secret_keys(cache[m], d, tr.nkeys[m], nullptr);
            }
            if (!rc && tr.pk[m]) {
                cudaDeviceSynchronize();
                cudaMemcpy(d, tr.pk[m], tr.nkeys[m] * p.pk_bytes, cudaMemcpyHostToDevice);
                rc = cudil_engine_set_public_keys(cache[m], d, tr.nkeys[m], nullptr);
            }
            cudaDeviceSynchronize();
            cudaFree(d);
            used_bytes += cudil_engine_device_bytes(cache[m]);
        }
    }
    if (rc) {
        cleanup();
        return rc;
    }
    if (cfg->device_budget_bytes && used_bytes > cfg->device_budget_bytes) {
        cleanup();
        return CUDIL_ERR_BUDGET;
    }

    // batch slots: round-robin over the lanes in use while the budget allows
    std::atomic<size_t> completed{0};
    std::vector<std::vector<Slot *>> lane_slots(6);
    std::vector<int> lanes;
    for (int m = 0; m < 3; ++m)
        for (int op = 0; op < 2; ++op) {
            bool any = false;
            for (size_t i = 0; i < nreq && !any; ++i) any = (mode_index(reqs[i].mode) == m && reqs[i].op == op);
            if (any) lanes.push_back(m * 2 + op);
        }
    // slots per lane: slots_per_lane each, or (lane_slots_by_load) in proportion to the lane's share
    // of the requests, never fewer than slots_per_lane
    std::vector<int> want(6, cfg->slots_per_lane);
    if (cfg->lane_slots_by_load && nreq) {
        std::vector<size_t> count(6, 0);
        for (size_t i = 0; i < nreq; ++i) ++count[mode_index(reqs[i].mode) * 2 + reqs[i].op];
        const double total_slots = (double)cfg->slots_per_lane * (double)lanes.size();
        for (int lane : lanes)
            want[lane] = std::max(cfg->slots_per_lane, (int)(total_slots * (double)count[lane] / (double)nreq + 0.5));
    }
    const int max_want = *std::max_element(want.begin(), want.end());
    for (int k = 0; k < max_want && rc == CUDIL_OK; ++k) {
        for (int lane : lanes) {
            if (k >= want[lane]) continue;
            const int m = lane / 2, op = lane % 2;
            size_t remaining = 0;
            if (cfg->device_budget_bytes) {
                if (used_bytes >= cfg->device_budget_bytes) {
                    if (k == 0) rc = CUDIL_ERR_BUDGET;  // every lane in use needs one slot
                    continue;
                }
                remaining = cfg->device_budget_bytes - used_bytes;
            }
            auto s = std::make_unique<Slot>();
            s->lane = lane;
            s->mode = kModes[m];
            s->op = op;
            s->completed = &completed;
            const int src = make_slot(*s, cfg, &tr, cache, remaining);
            if (src) {
                s->release();
                if (src == CUDIL_ERR_BUDGET && k > 0) continue;
                rc = src;
                break;
            }
            used_bytes += s->device_bytes;
            lane_slots[lane].push_back(s.get());
            slots.push_back(std::move(s));
        }
    }
    if (rc) {
        cleanup();
        return rc;
    }
    // warm-up: one batch of the lane's first request per slot, outside the replay clock
    for (auto &s : slots) {
        for (size_t i = 0; i < nreq; ++i)
            if (mode_index(reqs[i].mode) * 2 + reqs[i].op == s->lane) {
                s->batch.assign(1, (uint32_t)i);
                break;
            }
        rc = s->run_batch(false);
        s->batch.clear();
        if (rc) {
            cleanup();
            return rc;
        }
    }
    for (auto &s : slots) {
        Slot *sp = s.get();
        s->worker = std::thread([sp, device] { sp->loop(device); });
    }

    // ------------------------------------------------------------- replay
    std::vector<std::deque<uint32_t>> pending(6);
    tr.t0 = Clock::now();
    size_t next = 0;
    size_t launched_batches = 0;
    while (completed.load() < nreq) {
        const double now = std::chrono::duration<double>(Clock::now() - tr.t0).count();
        while (next < nreq && reqs[next].arrival_s <= now) {
            const cudil_request &r = reqs[next];
            pending[mode_index(r.mode) * 2 + r.op].push_back((uint32_t)next);
            ++next;
        }
        bool progressed = false;
        for (int lane : lanes) {
            auto &q = pending[lane];
            if (q.empty()) continue;
            for (Slot *s : lane_slots[lane]) {
                if (q.empty()) break;
                if (s->busy.load()) continue;
                if (s->error.load()) {
                    rc = s->error.load();
                    break;
                }
                const size_t take = std::min<size_t>(q.size(), (size_t)cfg->max_batch);
                {
                    // the slot is marked busy in the same locked region that publishes its work, so
                    // a worker that wakes at once (or spuriously) cannot finish and clear busy first
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->batch.assign(q.begin(), q.begin() + (long)take);
                    s->busy = true;
                    s->has_work = true;
                }
                q.erase(q.begin(), q.begin() + (long)take);
                s->cv.notify_one();
                ++launched_batches;
                progressed = true;
            }
            if (rc) break;
        }
        if (rc) break;
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    const double wall = std::chrono::duration<double>(Clock::now() - tr.t0).count();
    for (auto &s : slots)
        if (!rc && s->error.load()) rc = s->error.load();
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->wall_s = wall;
        stats->batches = launched_batches;
        stats->slots = slots.size();
        stats->device_bytes = used_bytes;
        for (auto &s : slots) {
            stats->host_stage_s += s->stage_ns.load() * 1e-9;
            stats->device_wait_s += s->device_ns.load() * 1e-9;
            stats->host_post_s += s->post_ns.load() * 1e-9;
        }
    }
    cleanup();
    return rc;
}
