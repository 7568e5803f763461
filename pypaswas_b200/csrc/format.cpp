// format.cpp -- trimmedFasta output of a hit set without Python Hit objects.
//
// The trimmer's output path of the reference builds a Hit per walk result
// (SmithWaterman._print_alignments, SmithWaterman.py:822-838), filters it
// (_filter_hit, :843-848), de-duplicates it in a HitList (HitList.append,
// HitList.py:28-52) and prints HitList.real_hits sorted by (query id, target
// id, score) as trimmedFasta records (Formatters.py:110-150,
// Hit.get_trimmed_line, Hit.py:274-286).  pw_trimmed_fasta does the same on
// the engine's hit records and writes the same bytes.  Ids are ranked by the
// caller (Python's string order), so ordering and de-duplication compare
// integers; the target ids arrive with the "_RC" suffix already stripped.
#include <algorithm>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "pw_host.h"

#include "../../include/paswas_b200.h"

namespace {

struct Key {
    int32_t q, t;
    int64_t a, b;
    bool operator==(const Key& o) const { return q == o.q && t == o.t && a == o.a && b == o.b; }
};

// splitmix64 finaliser over the four fields
inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct KeyHash {
    size_t operator()(const Key& k) const {
        const uint64_t ids = ((uint64_t)(uint32_t)k.q << 32) | (uint32_t)k.t;
        return (size_t)mix64(mix64(ids) ^ (uint64_t)k.a ^ ((uint64_t)k.b << 29) ^ ((uint64_t)k.b >> 35));
    }
};

// Open-addressing table Key -> int64 (linear probing, tombstones on erase).
struct FlatMap {
    std::vector<Key> keys;
    std::vector<int64_t> vals;
    std::vector<uint8_t> state;  // 0 empty, 1 used, 2 erased
    size_t mask = 0;
    explicit FlatMap(size_t n) {
        size_t cap = 16;
        while (cap < 2 * n + 16) cap <<= 1;
        keys.resize(cap);
        vals.resize(cap);
        state.assign(cap, 0);
        mask = cap - 1;
    }
    int64_t* find(const Key& k) {
        for (size_t i = KeyHash()(k) & mask;; i = (i + 1) & mask) {
            if (state[i] == 0) return nullptr;
            if (state[i] == 1 && keys[i] == k) return &vals[i];
        }
    }
    void put(const Key& k, int64_t v) {
        size_t slot = SIZE_MAX;
        for (size_t i = KeyHash()(k) & mask;; i = (i + 1) & mask) {
            if (state[i] == 0) {
                if (slot == SIZE_MAX) slot = i;
                break;
            }
            if (state[i] == 2) {
                if (slot == SIZE_MAX) slot = i;
            } else if (keys[i] == k) {
                vals[i] = v;
                return;
            }
        }
        keys[slot] = k;
        vals[slot] = v;
        state[slot] = 1;
    }
    void erase(const Key& k) {
        for (size_t i = KeyHash()(k) & mask;; i = (i + 1) & mask) {
            if (state[i] == 0) return;
            if (state[i] == 1 && keys[i] == k) {
                state[i] = 2;
                return;
            }
        }
    }
};

struct Rec {
    int32_t q, t;     // query / target list indices
    int32_t qr, tr;   // id ranks
    int64_t s0, t0;   // start of the hit (query, target), start positions added
    int64_t t1;       // end on the target
    double score;
};

}  // namespace

// Key -> int64 over a handful of entries: a linear scan (most (query,
// target) groups hold one or two hits).
struct SmallMap {
    std::vector<std::pair<Key, int64_t>> v;
    int64_t* find(const Key& k) {
        for (auto& e : v)
            if (e.first == k) return &e.second;
        return nullptr;
    }
    void put(const Key& k, int64_t x) {
        if (int64_t* f = find(k))
            *f = x;
        else
            v.push_back({k, x});
    }
    void erase(const Key& k) {
        for (size_t i = 0; i < v.size(); ++i)
            if (v[i].first == k) {
                v[i] = v.back();
                v.pop_back();
                return;
            }
    }
};

// HitList.append (HitList.py:28-52) over the hits of one (query id, target
// id) group in walk order: `best` maps a start or end key to its hit,
// `real_pos` a start key to its slot of `real` (Python's dict order: a new
// key goes last, a replaced one keeps its place, a deleted one is gone).
// Survivors go to `out` ordered by score, ties in slot order; returns their
// number.
template <typename Map>
static int64_t append_group(const pw_hit* hits, const Rec* rec, const int64_t* q_start_pos, const uint32_t* grp,
                            int64_t n, Map& best, Map& real_pos, std::vector<int64_t>& real, int64_t* out) {
    real.clear();
    for (int64_t g = 0; g < n; ++g) {
        const int64_t i = grp[g];
        const Rec& r = rec[i];
        const int64_t s1 = hits[i].s_end + q_start_pos[r.q];
        const Key k0{r.qr, r.tr, r.s0, r.t0}, k1{r.qr, r.tr, s1, r.t1};
        const int64_t* f0 = best.find(k0);
        const int64_t* f1 = best.find(k1);
        const bool better_end = f1 && rec[*f1].score < r.score;
        if ((!f0 && !f1) || better_end || (f0 && rec[*f0].score < r.score)) {
            if (better_end) {
                const Rec& o = rec[*f1];
                const Key ok{o.qr, o.tr, o.s0, o.t0};
                if (int64_t* slot = real_pos.find(ok)) {
                    real[*slot] = -1;
                    real_pos.erase(ok);
                }
            }
            best.put(k0, i);
            best.put(k1, i);
            if (int64_t* slot = real_pos.find(k0)) {
                real[*slot] = i;
            } else {
                real_pos.put(k0, (int64_t)real.size());
                real.push_back(i);
            }
        }
    }
    int64_t m = 0;
    for (int64_t i : real)
        if (i >= 0) out[m++] = i;
    std::stable_sort(out, out + m, [&](int64_t a, int64_t b) { return rec[a].score < rec[b].score; });
    return m;
}

// The driver's HitList for these records: locations checked as the Hit
// constructor checks them (Hit.py:16-60; any invalid one fails the call, as
// the reference's exception does), the filter (SmithWaterman._filter_hit),
// HitList.append in walk order, then HitList.real_hits sorted by (query id,
// target id, score), stable (Formatters.py:34-37).  Every key that
// HitList.append looks up carries the hit's two ids, so hits of different
// (query id, target id) groups never meet: the passing hits are grouped by
// their id ranks (a stable radix sort keeps walk order inside a group), the
// groups run the append rule independently on host threads, and the
// survivors come out in group order, by score inside a group, ties in the
// order their keys entered the dict.
static int ordered_real_hits(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                             const int32_t* q_rank, const int64_t* q_orig_len, const int64_t* q_start_pos,
                             const int32_t* t_rank, const int64_t* t_orig_len, const int64_t* t_start_pos,
                             const double* thresholds, std::vector<Rec>& rec, std::vector<int64_t>& order) {
    rec.resize((size_t)n_hits);
    std::vector<uint8_t> pass((size_t)n_hits, 0);
    std::atomic<bool> bad{false};
    int64_t max_tr = 0;
    for (int32_t t = 0; t < n_targets; ++t) max_tr = std::max<int64_t>(max_tr, t_rank[t]);
    parallel_for(n_hits, [&](int64_t i0, int64_t i1) {
        bool ok = true;
        for (int64_t i = i0; i < i1; ++i) {
            const pw_hit& h = hits[i];
            const int q = h.query, t = h.target;
            if (q < 0 || q >= n_queries || t < 0 || t >= n_targets) {
                ok = false;
                break;
            }
            const int64_t s0 = h.s_start + q_start_pos[q], s1 = h.s_end + q_start_pos[q];
            const int64_t t0 = h.t_start + t_start_pos[t], t1 = h.t_end + t_start_pos[t];
            if (!(0 <= s0 && s0 < s1 && s1 < q_orig_len[q] && 0 <= t0 && t0 < t1 && t1 < t_orig_len[t])) {
                ok = false;
                break;
            }
            const Rec r{q, t, q_rank[q], t_rank[t], s0, t0, t1, (double)h.score};
            rec[i] = r;
            // SmithWaterman._filter_hit
            const double span = (double)(s1 - s0 + 1);
            const double rel = r.score / (double)std::min(q_orig_len[q], t_orig_len[t]);
            const double ident = (double)h.matches / span;
            const double cov = span / (double)q_orig_len[q];
            const double base = r.score / (double)h.n_cols;
            pass[i] = rel >= thresholds[0] && ident >= thresholds[1] && cov >= thresholds[2] && base >= thresholds[3];
        }
        if (!ok) bad = true;
    }, 1 << 16);
    if (bad) return PW_ERR_ARG;
    std::vector<uint64_t> key;
    std::vector<uint32_t> hit_of;
    key.reserve((size_t)n_hits);
    hit_of.reserve((size_t)n_hits);
    for (int64_t i = 0; i < n_hits; ++i)
        if (pass[i]) {
            key.push_back((uint64_t)rec[i].qr * (uint64_t)(max_tr + 1) + (uint64_t)rec[i].tr);
            hit_of.push_back((uint32_t)i);
        }
    const int64_t m = (int64_t)key.size();
    std::vector<uint32_t> grp;  // passing hits, grouped, walk order inside a group
    {
        std::vector<uint64_t> k2 = key;
        const std::vector<uint32_t> o = radix_order(std::move(k2));
        grp.resize((size_t)m);
        for (int64_t k = 0; k < m; ++k) grp[k] = hit_of[o[k]];
        std::vector<uint64_t> ks((size_t)m);
        for (int64_t k = 0; k < m; ++k) ks[k] = key[o[k]];
        key.swap(ks);
    }
    std::vector<int64_t> gstart;
    for (int64_t k = 0; k < m; ++k)
        if (k == 0 || key[k] != key[k - 1]) gstart.push_back(k);
    const int64_t ng = (int64_t)gstart.size();
    gstart.push_back(m);
    std::vector<int64_t> surv((size_t)m), nsurv((size_t)ng);
    parallel_for(ng, [&](int64_t g0, int64_t g1) {
        SmallMap sb, sr;
        std::vector<int64_t> real;
        for (int64_t g = g0; g < g1; ++g) {
            const int64_t a = gstart[g], n = gstart[g + 1] - a;
            if (n == 1) {  // a lone hit is appended as it is
                surv[a] = grp[a];
                nsurv[g] = 1;
                continue;
            }
            if (n <= 32) {
                sb.v.clear();
                sr.v.clear();
                nsurv[g] = append_group(hits, rec.data(), q_start_pos, grp.data() + a, n, sb, sr, real, &surv[a]);
            } else {
                FlatMap fb((size_t)n * 2), fr((size_t)n);
                nsurv[g] = append_group(hits, rec.data(), q_start_pos, grp.data() + a, n, fb, fr, real, &surv[a]);
            }
        }
    }, 1 << 14);
    int64_t total = 0;
    for (int64_t g = 0; g < ng; ++g) total += nsurv[g];
    order.resize((size_t)total);
    int64_t w = 0;
    for (int64_t g = 0; g < ng; ++g)
        for (int64_t k = 0; k < nsurv[g]; ++k) order[w++] = surv[gstart[g] + k];
    return PW_OK;
}

extern "C" int pw_trimmed_fasta(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                                const int32_t* q_rank, const int64_t* q_orig_len,
                                const int64_t* q_start_pos, const char* q_id, const int64_t* q_id_off,
                                const char* q_seq, const int64_t* q_seq_off, const int32_t* t_rank,
                                const int64_t* t_orig_len, const int64_t* t_start_pos, const char* t_id,
                                const int64_t* t_id_off, const double* thresholds, char* out, int64_t out_cap,
                                int64_t* out_len) {
    if (n_hits < 0 || (n_hits > 0 && (!hits || !q_rank || !q_orig_len || !q_start_pos || !q_id || !q_id_off ||
                                      !q_seq || !q_seq_off || !t_rank || !t_orig_len || !t_start_pos || !t_id ||
                                      !t_id_off)) ||
        !thresholds || !out_len)
        return PW_ERR_ARG;
    std::vector<Rec> rec;
    std::vector<int64_t> order;
    const int rc = ordered_real_hits(hits, n_hits, n_queries, n_targets, q_rank, q_orig_len, q_start_pos, t_rank,
                                     t_orig_len, t_start_pos, thresholds, rec, order);
    if (rc != PW_OK) return rc;
    // ">" target id " " query id "\n" query[:t0] query[t1 + 1:] "\n": the
    // query cut by the hit's TARGET coordinates, as Hit.get_trimmed_line does;
    // record sizes, their offsets, then the records on host threads
    const int64_t m = (int64_t)order.size();
    std::vector<int64_t> at((size_t)m + 1, 0);
    for (int64_t k = 0; k < m; ++k) {
        const Rec& r = rec[order[k]];
        const int64_t L = q_seq_off[r.q + 1] - q_seq_off[r.q];
        const int64_t a = std::min(r.t0, L), b = std::min(r.t1 + 1, L);
        at[k + 1] = at[k] + 1 + (t_id_off[r.t + 1] - t_id_off[r.t]) + 1 + (q_id_off[r.q + 1] - q_id_off[r.q]) + 1 +
                    a + (L - b) + 1;
    }
    const int64_t need = at[m];
    *out_len = need;
    if (!out) return PW_OK;
    if (out_cap < need) return PW_ERR_CAPACITY;
    parallel_for(m, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) {
            const Rec& r = rec[order[k]];
            char* p = out + at[k];
            auto put = [&](const char* s, int64_t n) {
                if (n > 0) std::memcpy(p, s, (size_t)n);
                p += n;
            };
            const char* seq = q_seq + q_seq_off[r.q];
            const int64_t L = q_seq_off[r.q + 1] - q_seq_off[r.q];
            const int64_t a = std::min(r.t0, L), b = std::min(r.t1 + 1, L);
            *p++ = '>';
            put(t_id + t_id_off[r.t], t_id_off[r.t + 1] - t_id_off[r.t]);
            *p++ = ' ';
            put(q_id + q_id_off[r.q], q_id_off[r.q + 1] - q_id_off[r.q]);
            *p++ = '\n';
            put(seq, a);
            put(seq + b, L - b);
            *p++ = '\n';
        }
    }, 1 << 15);
    return PW_OK;
}

// Python's repr of a float (str(float) in Python 3): the shortest digits that
// round-trip (std::to_chars), laid out as Python's float_repr does --
// exponent form when the decimal point falls before the 4th leading zero or
// after the 16th digit, else fixed form, with ".0" after an integer value.
static void put_pyfloat(std::string& o, double v) {
    if (std::isnan(v)) {
        o += "nan";
        return;
    }
    if (std::isinf(v)) {
        o += v < 0 ? "-inf" : "inf";
        return;
    }
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof(buf) - 1, v, std::chars_format::scientific);
    *r.ptr = '\0';  // the exponent is read up to here
    const char* p = buf;
    if (*p == '-') {
        o += '-';
        ++p;
    }
    std::string digits(1, *p++);
    if (*p == '.') {
        ++p;
        while (*p != 'e') digits += *p++;
    }
    const int decpt = std::atoi(p + 1) + 1;  // value = 0.digits x 10^decpt
    const int n = (int)digits.size();
    if (decpt <= -4 || decpt > 16) {
        o += digits[0];
        if (n > 1) {
            o += '.';
            o.append(digits, 1, std::string::npos);
        }
        int e = decpt - 1;
        o += e < 0 ? "e-" : "e+";
        e = e < 0 ? -e : e;
        if (e < 10) o += '0';
        o += std::to_string(e);
    } else if (decpt <= 0) {
        o += "0.";
        o.append((size_t)(-decpt), '0');
        o += digits;
    } else if (decpt >= n) {
        o += digits;
        o.append((size_t)(decpt - n), '0');
        o += ".0";
    } else {
        o.append(digits, 0, (size_t)decpt);
        o += '.';
        o.append(digits, (size_t)decpt, std::string::npos);
    }
}

// TXT records (DefaultFormatter, Formatters.py:19-31) of the same HitList:
// "query, target, s_start, s_end, t_start, t_end, score, matches, mismatches,
// gaps, columns, score/columns, query length, target length, score/query
// length, score/target length, distance" and the three alignment strings,
// each record followed by a newline.  Only the record bytes differ from
// pw_trimmed_fasta's arguments: strbuf holds the hits' strings (pw_get_hits)
// and t_id the target ids as they are.
extern "C" int pw_txt_records(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                              const char* strbuf, int64_t strbuf_bytes, const int32_t* q_rank, const int64_t* q_orig_len, const int64_t* q_start_pos,
                              const char* q_id, const int64_t* q_id_off, const int32_t* t_rank,
                              const int64_t* t_orig_len, const int64_t* t_start_pos, const char* t_id,
                              const int64_t* t_id_off, const double* thresholds, char* out, int64_t out_cap,
                              int64_t* out_len) {
    if (n_hits < 0 || (n_hits > 0 && (!hits || !strbuf || !q_rank || !q_orig_len || !q_start_pos || !q_id ||
                                      !q_id_off || !t_rank || !t_orig_len || !t_start_pos || !t_id || !t_id_off)) ||
        !thresholds || !out_len)
        return PW_ERR_ARG;
    for (int64_t i = 0; i < n_hits; ++i)
        if (hits[i].n_cols < 0 || hits[i].str_offset < 0 || hits[i].str_offset + 3 * (int64_t)hits[i].n_cols > strbuf_bytes)
            return PW_ERR_ARG;
    std::vector<Rec> rec;
    std::vector<int64_t> order;
    const int rc = ordered_real_hits(hits, n_hits, n_queries, n_targets, q_rank, q_orig_len, q_start_pos, t_rank,
                                     t_orig_len, t_start_pos, thresholds, rec, order);
    if (rc != PW_OK) return rc;
    std::string o;
    for (int64_t i : order) {
        const pw_hit& h = hits[i];
        const Rec& r = rec[i];
        const int64_t n = h.n_cols;
        const int64_t s1 = h.s_end + q_start_pos[r.q];
        const int64_t ql = q_orig_len[r.q], tl = t_orig_len[r.t];
        o.append(q_id + q_id_off[r.q], (size_t)(q_id_off[r.q + 1] - q_id_off[r.q]));
        o += ", ";
        o.append(t_id + t_id_off[r.t], (size_t)(t_id_off[r.t + 1] - t_id_off[r.t]));
        for (int64_t v : {r.s0, s1, r.t0, r.t1}) {
            o += ", ";
            o += std::to_string(v);
        }
        o += ", ";
        put_pyfloat(o, r.score);
        for (int64_t v : {(int64_t)h.matches, (int64_t)h.mismatches, n - h.matches - h.mismatches, n}) {
            o += ", ";
            o += std::to_string(v);
        }
        o += ", ";
        put_pyfloat(o, r.score / (double)n);
        o += ", ";
        o += std::to_string(ql);
        o += ", ";
        o += std::to_string(tl);
        o += ", ";
        put_pyfloat(o, r.score / (double)ql);
        o += ", ";
        put_pyfloat(o, r.score / (double)tl);
        o += ", None\n";
        const char* sb = strbuf + h.str_offset;
        o.append(sb, (size_t)n);
        o += '\n';
        o.append(sb + n, (size_t)n);
        o += '\n';
        o.append(sb + 2 * n, (size_t)n);
        o += '\n';
    }
    *out_len = (int64_t)o.size();
    if (!out) return PW_OK;
    if (out_cap < (int64_t)o.size()) return PW_ERR_CAPACITY;
    if (!o.empty()) std::memcpy(out, o.data(), o.size());
    return PW_OK;
}

namespace {

// Python's identifier[:-3] if identifier[-2:] == "RC" else identifier
// (the formatters' RC suffix strip; Hit.py:159-164, Formatters.py:67-83)
inline bool ends_rc(const char* s, int64_t n) { return n >= 2 && s[n - 2] == 'R' && s[n - 1] == 'C'; }
inline int64_t stripped_len(const char* s, int64_t n) { return ends_rc(s, n) ? std::max<int64_t>(n - 3, 0) : n; }

// IUPAC complement (case kept): the table the reverse-complement targets use
struct Complement {
    char t[256];
    Complement() {
        for (int i = 0; i < 256; ++i) t[i] = (char)i;
        const char* from = "ACGTUNKMRYSWBDHVacgtunkmryswbdhv";
        const char* to = "TGCAANMKYRSWVHDBtgcaanmkyrswvhdb";
        for (int i = 0; from[i]; ++i) t[(uint8_t)from[i]] = to[i];
    }
};

}  // namespace

// SAM text (SamFormatter.print_results, Formatters.py:51-106) of the same
// HitList: "@HD", one "@SQ" line per target id in order of first use (the
// formatter's dict keyed by the id without its RC suffix, looked up by the id
// as it is), "@PG", then Hit.get_sam_line per hit (Hit.py:222-272,338-406):
// QNAME / RNAME without the RC suffix, FLAG 16 when either id ends in "RC",
// POS 1-based on the target (mirrored on RC hits), MAPQ 255, the extended
// CIGAR of the alignment string (reversed on RC hits, soft clips mirrored),
// SEQ the query (reverse-complemented on RC hits), then AS:i / RS:f / BS:f /
// QC:f / QI:f with Python's int() and float repr.  strbuf holds the hits'
// strings (pw_get_hits); ids arrive as they are.
extern "C" int pw_sam_records(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                              const char* strbuf, int64_t strbuf_bytes, const int32_t* q_rank,
                              const int64_t* q_orig_len, const int64_t* q_start_pos, const char* q_id,
                              const int64_t* q_id_off, const char* q_seq, const int64_t* q_seq_off,
                              const int32_t* t_rank, const int64_t* t_orig_len, const int64_t* t_start_pos,
                              const char* t_id, const int64_t* t_id_off, const double* thresholds, char* out,
                              int64_t out_cap, int64_t* out_len) {
    if (n_hits < 0 || (n_hits > 0 && (!hits || !strbuf || !q_rank || !q_orig_len || !q_start_pos || !q_id ||
                                      !q_id_off || !q_seq || !q_seq_off || !t_rank || !t_orig_len ||
                                      !t_start_pos || !t_id || !t_id_off)) ||
        !thresholds || !out_len)
        return PW_ERR_ARG;
    for (int64_t i = 0; i < n_hits; ++i)
        if (hits[i].n_cols <= 0 || hits[i].str_offset < 0 ||
            hits[i].str_offset + 3 * (int64_t)hits[i].n_cols > strbuf_bytes)
            return PW_ERR_ARG;
    std::vector<Rec> rec;
    std::vector<int64_t> order;
    const int rc = ordered_real_hits(hits, n_hits, n_queries, n_targets, q_rank, q_orig_len, q_start_pos, t_rank,
                                     t_orig_len, t_start_pos, thresholds, rec, order);
    if (rc != PW_OK) return rc;
    static const Complement comp;
    // @SQ lines: a dict keyed by the stripped id; a hit whose id is already a
    // key (an id without the suffix) is skipped, otherwise its stripped key is
    // (re)assigned, keeping the key's first position
    std::vector<std::string> sq;
    {
        std::unordered_map<std::string, size_t> keys;  // stripped id -> its line
        int prev = -1;
        for (int64_t i : order) {
            const int t = rec[i].t;
            if (t == prev) continue;  // the same lookup and assignment again: no change
            prev = t;
            const char* id = t_id + t_id_off[t];
            const int64_t n = t_id_off[t + 1] - t_id_off[t];
            if (keys.count(std::string(id, (size_t)n))) continue;
            const std::string key(id, (size_t)stripped_len(id, n));
            std::string line = "@SQ\tSN:" + key + "\tLN:" + std::to_string(t_orig_len[t]);
            auto f = keys.find(key);
            if (f != keys.end()) {
                sq[f->second] = std::move(line);
            } else {
                keys.emplace(key, sq.size());
                sq.push_back(std::move(line));
            }
        }
    }
    std::string o = "@HD\tVN:1.4\tSO:unknown\n";
    for (const std::string& l : sq) {
        o += l;
        o += '\n';
    }
    o += "@PG\tID:0\tPN:paswas\tVN:3.0\n";
    std::string aln, smatch;
    for (int64_t i : order) {
        const pw_hit& h = hits[i];
        const Rec& r = rec[i];
        const int64_t n = h.n_cols;
        const char* qi = q_id + q_id_off[r.q];
        const int64_t qn = q_id_off[r.q + 1] - q_id_off[r.q];
        const char* ti = t_id + t_id_off[r.t];
        const int64_t tn = t_id_off[r.t + 1] - t_id_off[r.t];
        const bool is_rc = ends_rc(qi, qn) || ends_rc(ti, tn);
        const int64_t s0 = r.s0, s1 = h.s_end + q_start_pos[r.q];
        const int64_t ql = q_orig_len[r.q], tl = t_orig_len[r.t];
        const char* seq = q_seq + q_seq_off[r.q];
        const int64_t L = q_seq_off[r.q + 1] - q_seq_off[r.q];
        const char* sb = strbuf + h.str_offset;
        smatch.assign(sb, (size_t)n);
        aln.assign(sb + n, (size_t)n);
        if (is_rc) {
            std::reverse(aln.begin(), aln.end());
            std::reverse(smatch.begin(), smatch.end());
        }
        o.append(qi, (size_t)stripped_len(qi, qn));
        o += is_rc ? "\t16\t" : "\t0\t";
        o.append(ti, (size_t)stripped_len(ti, tn));
        o += '\t';
        o += std::to_string(is_rc ? tl - r.t1 : r.t0 + 1);
        o += "\t255\t";
        // CIGAR: soft clip, one run per stretch of equal alignment
        // characters named by its last column, soft clip
        if (is_rc) {
            o += std::to_string(L - s1 - 1);
            o += 'S';
        } else if (s0 > 0) {
            o += std::to_string(s0);
            o += 'S';
        }
        auto cigar_char = [&](int64_t p) -> char {
            if (aln[p] == '|') return '=';
            if (aln[p] == '.') return 'X';
            return smatch[p] == '-' ? 'D' : 'I';
        };
        int64_t run = 0;
        for (int64_t k = 1; k < n; ++k)
            if (aln[k] != aln[run]) {
                o += std::to_string(k - run);
                o += cigar_char(k - 1);
                run = k;
            }
        o += std::to_string(n - run);
        o += cigar_char(n - 1);
        const int64_t tail = is_rc ? s0 : ql - s1 - 1;
        if (tail > 0) {
            o += std::to_string(tail);
            o += 'S';
        }
        o += "\t*\t0\t0\t";
        if (is_rc) {
            for (int64_t k = L - 1; k >= 0; --k) o += comp.t[(uint8_t)seq[k]];
        } else {
            o.append(seq, (size_t)L);
        }
        o += "\t*\tAS:i:";
        o += std::to_string((int64_t)r.score);
        const double span = (double)(s1 - s0 + 1);
        o += "\tRS:f:";
        put_pyfloat(o, r.score / (double)std::min(ql, tl));
        o += "\tBS:f:";
        put_pyfloat(o, r.score / (double)n);
        o += "\tQC:f:";
        put_pyfloat(o, span / (double)ql);
        o += "\tQI:f:";
        put_pyfloat(o, (double)h.matches / span);
        o += '\n';
    }
    *out_len = (int64_t)o.size();
    if (!out) return PW_OK;
    if (out_cap < (int64_t)o.size()) return PW_ERR_CAPACITY;
    if (!o.empty()) std::memcpy(out, o.data(), o.size());
    return PW_OK;
}
