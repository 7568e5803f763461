// server.cpp -- the serving loop: continuous batching of alignment requests
// against a database kept resident on the device.
//
// No counterpart in the reference (pyPaSWAS runs one batch per process).  It is
// built from the engine's own entry points (pw_set_queries / pw_align / ...),
// so every request gets exactly the result a lone pw_align of that query
// against the database gives.
//
// Structure: W worker threads, each owning one engine (its own CUDA stream and
// device buffers) with the database loaded once.  A free worker takes the
// requests that are waiting -- those that arrived while the other workers' batches
// were on the GPU -- up to `max_batch` of either mode, and runs them as one batch
// (the full path when one of them wants its hits);
// batches of different workers overlap on the device.  Traceback requests are
// admitted by direction-matrix memory: each reserves an estimate of its cell-code
// bytes from a shared budget (query length x database residues x the traced
// fraction observed so far), a batch starts only when its reservation fits, and
// the engine's memory waves keep the batch's cell codes within the reservation.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/paswas_b200.h"

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t ticket = 0;
    std::vector<uint8_t> residues;
    int32_t mode = PW_SERVE_TOP;
    int32_t top_k = 10;
    int64_t est_bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    bool done = false;
    int32_t status = PW_OK;
    std::string error;
    int32_t batch_queries = 0, worker = -1;
    int64_t cells = 0, reserved = 0;
    double score_kernel_ms = 0, setup_ms = 0, call_ms = 0;
    std::vector<int32_t> top_targets;
    std::vector<float> top_scores;
    std::vector<pw_hit> hits;
    std::vector<char> strings;
};

struct Worker {
    pw_engine* engine = nullptr;
    std::thread thread;
};

}  // namespace

struct pw_server {
    int device = 0;
    int max_batch = 16;
    int policy = 1;              // PW_SERVE_TUNE_POLICY (shortest first with aging)
    double age_ms = 25.0;        // PW_SERVE_TUNE_AGE_MS
    int64_t max_residues = 0;    // PW_SERVE_TUNE_MAX_RESIDUES (0: no limit)
    int64_t budget = 0;          // direction-matrix bytes shared by all traceback batches
    int64_t in_use = 0;          // reserved by running batches
    int64_t peak_in_use = 0;
    double traced_fraction = 1e-3;  // running estimate: traced cells / cells of traceback batches
    std::vector<Worker> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::unordered_map<int64_t, Request*> requests;
    int64_t next_ticket = 1;
    bool stopping = false;
    bool ready = false;          // scoring and database loaded
    int64_t db_residues = 0;
    int32_t db_n = 0;
    std::string err;
    // statistics
    int64_t submitted = 0, completed = 0, batches = 0, cells = 0;
    double busy_ms = 0;
};

namespace {

int server_fail(pw_server* s, int code, const std::string& msg) {
    std::lock_guard<std::mutex> g(s->mu);
    s->err = msg;
    return code;
}

// Takes the next batch: requests in queue order (arrival order, or shortest
// first under policy 1) up to max_batch, of either mode.  A batch with a
// traceback request runs the full path with a trace mask that leaves the
// top-k requests' pairs at their maxima (pw_set_query_trace), so only
// traceback requests reserve their direction-memory estimate from the shared
// budget; one joins only while the reservations fit the free budget (the
// first one alone may take the whole budget when nothing else is reserved),
// and one that does not fit leaves the batch to the requests behind it.
// Called with s->mu held.
std::vector<Request*> take_batch(pw_server* s, int64_t* reserve) {
    std::vector<Request*> batch;
    *reserve = 0;
    if (s->pending.empty()) return batch;
    if (s->policy == 1) {
        // shortest first, requests past the age limit first of all (oldest
        // first among them): the pending queue is reordered that way, and
        // the batch is then taken from its front
        const double now = now_ms();
        std::vector<Request*> v(s->pending.begin(), s->pending.end());
        std::stable_sort(v.begin(), v.end(), [&](const Request* a, const Request* b) {
            const bool oa = now - a->t_submit >= s->age_ms, ob = now - b->t_submit >= s->age_ms;
            if (oa != ob) return oa;
            if (oa) return a->t_submit < b->t_submit;
            return a->residues.size() < b->residues.size();
        });
        s->pending.assign(v.begin(), v.end());
    }
    const int64_t free_b = s->budget - s->in_use;
    bool traceback = false;
    int64_t residues = 0;
    for (auto it = s->pending.begin(); it != s->pending.end() && (int)batch.size() < s->max_batch;) {
        Request* r = *it;
        if (s->max_residues > 0 && !batch.empty() && residues + (int64_t)r->residues.size() > s->max_residues) {
            ++it;  // would make the batch too long a run for the requests in it
            continue;
        }
        if (r->mode == PW_SERVE_TRACEBACK) {
            const int64_t need = std::min(r->est_bytes, s->budget);
            const bool alone = *reserve == 0 && s->in_use == 0;
            if (!alone && *reserve + need > free_b) {
                ++it;  // no room for it now
                continue;
            }
            *reserve += need;
            traceback = true;
        }
        batch.push_back(r);
        residues += (int64_t)r->residues.size();
        it = s->pending.erase(it);
    }
    *reserve = traceback ? std::max<int64_t>(std::min(*reserve, s->budget), 1) : 0;
    return batch;
}

void run_batch(pw_server* s, int w, pw_engine* e, std::vector<Request*>& batch, int64_t reserve) {
    const int n = (int)batch.size();
    // the full path when any request wants its hits, else score only
    int mode = PW_SERVE_TOP;
    for (const Request* r : batch)
        if (r->mode == PW_SERVE_TRACEBACK) mode = PW_SERVE_TRACEBACK;
    std::vector<int64_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (int64_t)batch[i]->residues.size();
    std::vector<uint8_t> res((size_t)std::max<int64_t>(off[n], 1));
    for (int i = 0; i < n; ++i)
        if (!batch[i]->residues.empty())
            std::memcpy(res.data() + off[i], batch[i]->residues.data(), batch[i]->residues.size());
    std::vector<int32_t> keys(n, -1);  // database keys are >= 0: no pair is skipped
    pw_run_info info;
    std::memset(&info, 0, sizeof(info));
    int rc = pw_set_queries(e, res.data(), off.data(), n, keys.data());
    if (rc == PW_OK && mode == PW_SERVE_TRACEBACK) {
        // only the traceback requests' pairs are traced
        std::vector<uint8_t> mask(n);
        bool all = true;
        for (int i = 0; i < n; ++i) {
            mask[i] = batch[i]->mode == PW_SERVE_TRACEBACK ? 1 : 0;
            all = all && mask[i];
        }
        if (!all) rc = pw_set_query_trace(e, mask.data(), n);
        if (rc == PW_OK) rc = pw_set_wave_limit(e, reserve);
    }
    if (rc == PW_OK) rc = pw_align(e, mode == PW_SERVE_TOP ? PW_FLAG_SCORE_ONLY : 0u, -1, &info);
    std::vector<float> pmax;
    std::vector<pw_hit> hits;
    std::vector<char> strings;
    bool any_top = false;
    for (const Request* r : batch) any_top = any_top || r->mode == PW_SERVE_TOP;
    if (rc == PW_OK && any_top) {
        pmax.resize((size_t)n * s->db_n);
        rc = pw_get_pair_max(e, pmax.data(), (int64_t)pmax.size());
    }
    if (rc == PW_OK && mode == PW_SERVE_TRACEBACK) {
        hits.resize((size_t)info.hits);
        strings.resize((size_t)std::max<int64_t>(info.string_bytes, 1));
        rc = pw_get_hits(e, hits.data(), info.hits, strings.data(), info.string_bytes);
    }
    const std::string msg = rc == PW_OK ? std::string() : std::string(pw_last_error(e));
    // top hits of the score-only requests: one host thread per request
    if (rc == PW_OK && any_top) {
        auto top = [&](int i) {
            Request* r = batch[i];
            if (r->mode != PW_SERVE_TOP) return;
            const float* row = pmax.data() + (size_t)i * s->db_n;
            std::vector<int32_t> idx(s->db_n);
            for (int32_t t = 0; t < s->db_n; ++t) idx[t] = t;
            const int k = std::min<int>(r->top_k, s->db_n);
            auto better = [&](int32_t a, int32_t b) { return row[a] > row[b] || (row[a] == row[b] && a < b); };
            std::partial_sort(idx.begin(), idx.begin() + k, idx.end(), better);
            r->top_targets.assign(idx.begin(), idx.begin() + k);
            r->top_scores.resize(k);
            for (int j = 0; j < k; ++j) r->top_scores[j] = row[idx[j]];
        };
        if (n == 1) {
            top(0);
        } else {
            std::vector<std::thread> th;
            th.reserve(n);
            for (int i = 0; i < n; ++i) th.emplace_back(top, i);
            for (auto& t : th) t.join();
        }
    }
    // per-request results
    for (int i = 0; i < n; ++i) {
        Request* r = batch[i];
        r->status = rc;
        r->error = msg;
        r->batch_queries = n;
        r->worker = w;
        r->cells = (int64_t)r->residues.size() * s->db_residues;
        r->reserved = mode == PW_SERVE_TRACEBACK ? reserve : 0;
        r->score_kernel_ms = info.score_kernel_ms;
        r->setup_ms = info.setup_ms;
        r->call_ms = info.total_ms;
        if (rc != PW_OK) continue;
        if (r->mode == PW_SERVE_TOP) {
            // filled above
        } else {
            for (const pw_hit& h : hits) {
                if (h.query != i) continue;
                pw_hit c = h;
                c.query = 0;
                c.str_offset = (int64_t)r->strings.size();
                r->strings.insert(r->strings.end(), strings.begin() + h.str_offset,
                                  strings.begin() + h.str_offset + 3 * (int64_t)h.n_cols);
                r->hits.push_back(c);
            }
        }
    }
    const double t = now_ms();
    std::lock_guard<std::mutex> g(s->mu);
    if (reserve > 0) {
        s->in_use -= reserve;
        if (rc == PW_OK && info.cells > 0) {
            const double f = (double)info.traced_cells / (double)info.cells;
            s->traced_fraction = 0.8 * s->traced_fraction + 0.2 * std::max(f, 1e-6);
        }
    }
    for (Request* r : batch) {
        r->t_done = t;
        r->done = true;
        s->cells += r->cells;
    }
    s->completed += n;
    s->batches += 1;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

void worker_loop(pw_server* s, int w) {
    pw_engine* e = s->workers[w].engine;
    for (;;) {
        std::vector<Request*> batch;
        int64_t reserve = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stopping && s->pending.empty()) return;
                if (s->ready) {
                    batch = take_batch(s, &reserve);
                    if (!batch.empty()) break;
                }
                s->cv_work.wait(lk);
            }
            const double t = now_ms();
            for (Request* r : batch) r->t_admit = t;
            if (reserve > 0) {
                s->in_use += reserve;
                s->peak_in_use = std::max(s->peak_in_use, s->in_use);
            }
        }
        const double t0 = now_ms();
        run_batch(s, w, e, batch, reserve);
        std::lock_guard<std::mutex> g(s->mu);
        s->busy_ms += now_ms() - t0;
    }
}

}  // namespace

extern "C" int pw_server_create(int device, int n_workers, int max_batch, int64_t direction_budget,
                                pw_server** out) {
    if (!out) return PW_ERR_ARG;
    *out = nullptr;
    if (n_workers < 1 || n_workers > 16 || max_batch < 1 || max_batch > 4096 || direction_budget < 0)
        return PW_ERR_ARG;
    pw_server* s = new pw_server();
    s->device = device;
    s->max_batch = max_batch;
    s->budget = direction_budget > 0 ? direction_budget : ((int64_t)8 << 30);
    for (int w = 0; w < n_workers; ++w) {
        pw_engine* e = nullptr;
        const int rc = pw_create(device, &e);
        if (rc != PW_OK) {
            for (Worker& x : s->workers) pw_destroy(x.engine);
            delete s;
            return rc;
        }
        Worker wk;
        wk.engine = e;
        s->workers.push_back(std::move(wk));
    }
    for (int w = 0; w < n_workers; ++w) s->workers[w].thread = std::thread(worker_loop, s, w);
    *out = s;
    return PW_OK;
}

extern "C" void pw_server_destroy(pw_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stopping = true;
        if (!s->ready) s->pending.clear();
    }
    s->cv_work.notify_all();
    for (Worker& w : s->workers)
        if (w.thread.joinable()) w.thread.join();
    for (Worker& w : s->workers) pw_destroy(w.engine);
    for (auto& kv : s->requests) delete kv.second;
    delete s;
}

extern "C" const char* pw_server_last_error(pw_server* s) {
    if (!s) return "no server";
    std::lock_guard<std::mutex> g(s->mu);
    return s->err.c_str();
}

extern "C" int pw_server_set_scoring(pw_server* s, const float* matrix, int dim, int char_offset, float gap, float ext,
                                     int affine, float lower_limit, float minimum_score, double host_minimum,
                                     double highest, double filter_factor) {
    if (!s) return PW_ERR_ARG;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->ready) {
            s->err = "scoring must be set before the database is loaded";
            return PW_ERR_STATE;
        }
    }
    for (Worker& w : s->workers) {
        const int rc = pw_set_scoring(w.engine, matrix, dim, char_offset, gap, ext, affine, lower_limit,
                                      minimum_score, host_minimum, highest, filter_factor);
        if (rc != PW_OK) return server_fail(s, rc, pw_last_error(w.engine));
    }
    return PW_OK;
}

extern "C" int pw_server_tune(pw_server* s, int key, int64_t value) {
    if (!s) return PW_ERR_ARG;
    if (key >= PW_SERVE_TUNE_POLICY) {
        std::lock_guard<std::mutex> g(s->mu);
        if (key == PW_SERVE_TUNE_POLICY && (value == 0 || value == 1)) {
            s->policy = (int)value;
        } else if (key == PW_SERVE_TUNE_AGE_MS && value >= 0) {
            s->age_ms = (double)value;
        } else if (key == PW_SERVE_TUNE_MAX_BATCH && value >= 1 && value <= 4096) {
            s->max_batch = (int)value;
        } else if (key == PW_SERVE_TUNE_MAX_RESIDUES && value >= 0) {
            s->max_residues = value;
        } else {
            s->err = "unknown server setting or value out of range";
            return PW_ERR_ARG;
        }
        return PW_OK;
    }
    for (Worker& w : s->workers) {
        const int rc = pw_set_tuning(w.engine, key, value);
        if (rc != PW_OK) return server_fail(s, rc, pw_last_error(w.engine));
    }
    return PW_OK;
}

extern "C" int pw_server_load_db(pw_server* s, const uint8_t* residues, const int64_t* offsets, int32_t n,
                                 const int32_t* id_keys) {
    if (!s) return PW_ERR_ARG;
    if (n <= 0 || !offsets || !id_keys) return server_fail(s, PW_ERR_ARG, "the database needs at least one sequence");
    for (int32_t i = 0; i < n; ++i)
        if (id_keys[i] < 0) return server_fail(s, PW_ERR_ARG, "database id keys must be >= 0");
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->ready) {
            s->err = "the database is already loaded";
            return PW_ERR_STATE;
        }
    }
    // every worker engine holds the database resident; a one-residue query
    // run prepares the device copy now instead of on the first request
    const uint8_t probe = residues ? residues[0] : 0;
    const int64_t poff[2] = {0, 1};
    const int32_t pkey = -1;
    for (Worker& w : s->workers) {
        int rc = pw_set_targets(w.engine, residues, offsets, n, id_keys);
        if (rc == PW_OK) rc = pw_set_queries(w.engine, &probe, poff, 1, &pkey);
        pw_run_info info;
        if (rc == PW_OK) rc = pw_align(w.engine, PW_FLAG_SCORE_ONLY, -1, &info);
        if (rc != PW_OK) return server_fail(s, rc, pw_last_error(w.engine));
    }
    // warm-up: one full-size batch per worker and mode (database sequences as
    // queries, so the traceback run walks their self-alignments), so that the
    // engines' device buffers have grown before the first request arrives
    {
        const int m = std::min<int>(s->max_batch, n);
        std::vector<int64_t> woff(m + 1, 0);
        for (int i = 0; i < m; ++i) woff[i + 1] = woff[i] + (offsets[i + 1] - offsets[i]);
        std::vector<int32_t> wkey(m, -1);
        for (Worker& w : s->workers) {
            int rc = pw_set_queries(w.engine, residues, woff.data(), m, wkey.data());
            pw_run_info info;
            if (rc == PW_OK) rc = pw_align(w.engine, PW_FLAG_SCORE_ONLY, -1, &info);
            if (rc == PW_OK) rc = pw_set_wave_limit(w.engine, std::min<int64_t>(s->budget, (int64_t)1 << 30));
            if (rc == PW_OK) rc = pw_align(w.engine, 0u, -1, &info);
            if (rc != PW_OK) return server_fail(s, rc, pw_last_error(w.engine));
        }
    }
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->db_n = n;
        s->db_residues = offsets[n];
        s->ready = true;
    }
    s->cv_work.notify_all();
    return PW_OK;
}

extern "C" int pw_server_submit(pw_server* s, const uint8_t* residues, int64_t length, int32_t mode, int32_t top_k,
                                int64_t* ticket) {
    if (!s || !ticket) return PW_ERR_ARG;
    if (length <= 0 || !residues) return server_fail(s, PW_ERR_ARG, "empty query");
    if (length > (1 << 24)) return server_fail(s, PW_ERR_ARG, "query longer than 16M residues");
    if (mode != PW_SERVE_TOP && mode != PW_SERVE_TRACEBACK) return server_fail(s, PW_ERR_ARG, "unknown mode");
    if (mode == PW_SERVE_TOP && top_k < 1) return server_fail(s, PW_ERR_ARG, "top_k must be >= 1");
    Request* r = new Request();
    r->residues.assign(residues, residues + length);
    r->mode = mode;
    r->top_k = top_k;
    r->t_submit = now_ms();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (!s->ready || s->stopping) {
            delete r;
            s->err = s->stopping ? "the server is stopping" : "the database is not loaded";
            return PW_ERR_STATE;
        }
        r->ticket = s->next_ticket++;
        r->est_bytes = std::max<int64_t>((int64_t)((double)length * (double)s->db_residues * s->traced_fraction * 2.0),
                                         (int64_t)16 << 20);
        s->requests[r->ticket] = r;
        s->pending.push_back(r);
        s->submitted++;
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return PW_OK;
}

extern "C" int pw_server_wait(pw_server* s, int64_t ticket, int32_t timeout_ms, pw_request_info* info) {
    if (!s) return PW_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) {
        s->err = "unknown ticket";
        return PW_ERR_ARG;
    }
    Request* r = it->second;
    const auto pred = [&] { return r->done; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
        return PW_ERR_TIMEOUT;
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->status = r->status;
        info->mode = r->mode;
        info->batch_queries = r->batch_queries;
        info->worker = r->worker;
        info->cells = r->cells;
        info->n_hits = r->mode == PW_SERVE_TOP ? (int64_t)r->top_targets.size() : (int64_t)r->hits.size();
        info->string_bytes = (int64_t)r->strings.size();
        info->reserved_bytes = r->reserved;
        info->queue_ms = r->t_admit - r->t_submit;
        info->run_ms = r->t_done - r->t_admit;
        info->latency_ms = r->t_done - r->t_submit;
        info->batch_score_kernel_ms = r->score_kernel_ms;
        info->batch_setup_ms = r->setup_ms;
        info->batch_call_ms = r->call_ms;
    }
    if (r->status != PW_OK) s->err = r->error;
    return r->status;
}

extern "C" int pw_server_top_hits(pw_server* s, int64_t ticket, int32_t* targets, float* scores, int32_t k) {
    if (!s) return PW_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second->done) {
        s->err = "unknown or unfinished ticket";
        return PW_ERR_STATE;
    }
    const Request* r = it->second;
    if (r->mode != PW_SERVE_TOP || k < (int32_t)r->top_targets.size()) {
        s->err = "not a top-hits request, or k smaller than its result";
        return PW_ERR_ARG;
    }
    for (size_t j = 0; j < r->top_targets.size(); ++j) {
        targets[j] = r->top_targets[j];
        scores[j] = r->top_scores[j];
    }
    return PW_OK;
}

extern "C" int pw_server_hits(pw_server* s, int64_t ticket, pw_hit* hits, int64_t max_hits, char* strbuf,
                              int64_t strbuf_bytes) {
    if (!s) return PW_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second->done) {
        s->err = "unknown or unfinished ticket";
        return PW_ERR_STATE;
    }
    const Request* r = it->second;
    if (max_hits < (int64_t)r->hits.size() || strbuf_bytes < (int64_t)r->strings.size()) {
        s->err = "result buffers too small";
        return PW_ERR_ARG;
    }
    if (!r->hits.empty()) std::memcpy(hits, r->hits.data(), r->hits.size() * sizeof(pw_hit));
    if (!r->strings.empty()) std::memcpy(strbuf, r->strings.data(), r->strings.size());
    return PW_OK;
}

extern "C" int pw_server_release(pw_server* s, int64_t ticket) {
    if (!s) return PW_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second->done) {
        s->err = "unknown or unfinished ticket";
        return PW_ERR_STATE;
    }
    delete it->second;
    s->requests.erase(it);
    return PW_OK;
}

extern "C" int pw_server_stats(pw_server* s, pw_server_counters* st) {
    if (!s || !st) return PW_ERR_ARG;
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->batches = s->batches;
    st->cells = s->cells;
    st->pending = (int64_t)s->pending.size();
    st->budget_bytes = s->budget;
    st->reserved_bytes = s->in_use;
    st->peak_reserved_bytes = s->peak_in_use;
    st->busy_ms = s->busy_ms;
    st->traced_fraction = s->traced_fraction;
    return PW_OK;
}
