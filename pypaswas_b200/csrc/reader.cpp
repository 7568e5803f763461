// reader.cpp -- FASTA / FASTQ records into packed buffers (host only).
//
// Replaces, for the engine's input, the reference's record preparation:
// BioPythonReader.read_records (pyPaSWAS/Core/Readers.py:90-118: SeqIO.parse,
// islice(start, end), the limit_length filter, SWSeqRecord's upper-casing,
// SWSeqRecord.py:16), complement_records / complement_records_only /
// reverse_records (Readers.py:68-86, the "_RC" ids) and sort_records
// (Readers.py:30-34, a stable sort by length, longest first).  The result is one
// residue array with offsets and one id array with offsets -- what
// pw_set_queries / pw_set_targets take -- with no per-record objects.
//
// Parsing follows Biopython's readers as pyPaSWAS uses them:
//   FASTA  text before the first '>' line is skipped; a record's title is its
//          '>' line without the '>' and without trailing whitespace; its id is
//          the title's first whitespace-separated word ("" for an empty title);
//          its sequence is its other lines, each without trailing whitespace,
//          joined, with spaces and carriage returns removed.
//   FASTQ  '@' title line, sequence lines up to a '+' line, then quality lines
//          until the quality is as long as the sequence; a record whose
//          quality length differs from its sequence length is an error.
// Line ends may be "\n" or "\r\n" (the reference opens files in universal
// newline mode).
#include <algorithm>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/paswas_b200.h"
#include "pw_host.h"

namespace {

int report(char* err, int32_t err_bytes, int code, const char* fmt, ...) {
    if (err && err_bytes > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, (size_t)err_bytes, fmt, ap);
        va_end(ap);
    }
    return code;
}

// One record as parsed: title id span in the input, sequence in a parser
// buffer (seq_begin there; `s` points at it once parsing is done).
struct Rec {
    int64_t id_begin, id_len;
    int64_t seq_begin, seq_len;
    const uint8_t* s;
};

}  // namespace

// Parsed records in their output order.  The residues are written by
// pw_records_copy straight from the parse buffers into the caller's array
// (upper-cased, complemented or reversed on the way); ids and offsets are
// built at parse time.
struct pw_records {
    std::vector<std::vector<uint8_t>> bufs;  // parsed sequence bytes (Rec::s points here)
    std::vector<Rec> recs;
    std::vector<int64_t> src;                // output record -> parsed record, in output order
    std::vector<uint8_t> kind;               // 0 as read, 1 reverse complement, 2 reversed
    std::vector<int64_t> off;
    std::vector<char> ids;
    std::vector<int64_t> id_off;
    int64_t dropped = 0;  // records removed by the length limit
};

namespace {

struct Lines {
    const char* p;
    const char* end;
    // next line without its line end; false at the end of the input
    bool next(const char*& b, const char*& e) {
        if (p >= end) return false;
        b = p;
        const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
        e = nl ? nl : end;
        p = nl ? nl + 1 : end;
        return true;
    }
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Python's str.rstrip() and the first word of str.split()
inline const char* rstrip(const char* b, const char* e) {
    while (e > b && is_space(e[-1])) --e;
    return e;
}

void first_word(const char* b, const char* e, int64_t& wb, int64_t& wl, const char* base) {
    while (b < e && is_space(*b)) ++b;
    const char* w = b;
    while (w < e && !is_space(*w)) ++w;
    wb = b - base;
    wl = w - b;
}

// appends a sequence line: spaces and carriage returns removed
inline void append_seq(std::vector<uint8_t>& seq, const char* b, const char* e) {
    while (b < e) {
        const char* c = b;
        while (c < e && *c != ' ' && *c != '\r') ++c;
        seq.insert(seq.end(), (const uint8_t*)b, (const uint8_t*)c);  // the run up to the next removed byte
        b = c < e ? c + 1 : e;
    }
}

// FASTA records of data[b0, b1) (ids as offsets into `data`).
int parse_fasta_range(const char* data, int64_t b0, int64_t b1, std::vector<Rec>& recs, std::vector<uint8_t>& seq) {
    Lines L{data + b0, data + b1};
    seq.reserve((size_t)(b1 - b0));
    const char *b, *e;
    bool in_rec = false;
    while (L.next(b, e)) {
        if (b < e && *b == '>') {
            if (in_rec) recs.back().seq_len = (int64_t)seq.size() - recs.back().seq_begin;
            Rec r;
            const char* te = rstrip(b + 1, e);
            first_word(b + 1, te, r.id_begin, r.id_len, data);
            r.seq_begin = (int64_t)seq.size();
            r.seq_len = 0;
            recs.push_back(r);
            in_rec = true;
        } else if (in_rec) {
            append_seq(seq, b, rstrip(b, e));
        }
    }
    if (in_rec) recs.back().seq_len = (int64_t)seq.size() - recs.back().seq_begin;
    return PW_OK;
}

// A whole FASTA input, in pieces on host threads: a piece starts at a line
// that begins with '>' (every such line starts a record, so the pieces parse
// independently); text before the first record is skipped as in one piece.
int parse_fasta(const char* data, int64_t n, std::vector<Rec>& recs, std::vector<std::vector<uint8_t>>& bufs) {
    const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    const int64_t pieces = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(hw, 32), n >> 22));
    std::vector<int64_t> cut{0};
    for (int64_t k = 1; k < pieces; ++k) {
        int64_t c = std::max(n * k / pieces, cut.back());
        // the next "\n>" at or after c: the '>' line starts the piece
        while (c < n) {
            const char* nl = (const char*)memchr(data + c, '\n', (size_t)(n - c));
            if (!nl) {
                c = n;
                break;
            }
            c = nl - data + 1;
            if (c < n && data[c] == '>') break;
        }
        cut.push_back(std::min(c, n));
    }
    cut.push_back(n);
    const int np = (int)cut.size() - 1;
    std::vector<std::vector<Rec>> pr((size_t)np);
    bufs.assign((size_t)np, {});
    parallel_for(np, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) parse_fasta_range(data, cut[k], cut[k + 1], pr[k], bufs[k]);
    }, 1);
    size_t total = 0;
    for (auto& v : pr) total += v.size();
    recs.clear();
    recs.reserve(total);
    for (int k = 0; k < np; ++k)
        for (Rec r : pr[k]) {
            r.s = bufs[k].data() + r.seq_begin;
            recs.push_back(r);
        }
    return PW_OK;
}

int parse_fastq(const char* data, int64_t n, std::vector<Rec>& recs, std::vector<uint8_t>& seq, char* err,
                int32_t err_bytes) {
    Lines L{data, data + n};
    const char *b, *e;
    // blank lines before the first record are skipped
    bool have = false;
    while (L.next(b, e)) {
        if (rstrip(b, e) != b) {
            have = true;
            break;
        }
    }
    while (have) {
        if (*b != '@')
            return report(err, err_bytes, PW_ERR_ARG, "FASTQ record does not start with '@' (record %zu)",
                          recs.size() + 1);
        Rec r;
        first_word(b + 1, rstrip(b + 1, e), r.id_begin, r.id_len, data);
        r.seq_begin = (int64_t)seq.size();
        bool plus = false;
        while (L.next(b, e)) {
            if (b < e && *b == '+') {
                plus = true;
                break;
            }
            append_seq(seq, b, rstrip(b, e));
        }
        if (!plus) return report(err, err_bytes, PW_ERR_ARG, "FASTQ record without a '+' line");
        r.seq_len = (int64_t)seq.size() - r.seq_begin;
        int64_t qlen = 0;
        have = false;
        while (qlen < r.seq_len && L.next(b, e)) {
            const char* qe = rstrip(b, e);
            qlen += qe - b;
        }
        if (qlen != r.seq_len)
            return report(err, err_bytes, PW_ERR_ARG, "FASTQ quality length %lld differs from sequence length %lld",
                          (long long)qlen, (long long)r.seq_len);
        recs.push_back(r);
        while (L.next(b, e)) {
            if (rstrip(b, e) != b) {
                have = true;
                break;
            }
        }
    }
    return PW_OK;
}

// IUPAC complement (case kept), the table the reverse-complement targets use
struct ComplementTable {
    uint8_t t[256];
    ComplementTable() {
        for (int i = 0; i < 256; ++i) t[i] = (uint8_t)i;
        const char* from = "ACGTUNKMRYSWBDHVacgtunkmryswbdhv";
        const char* to = "TGCAANMKYRSWVHDBtgcaanmkyrswvhdb";
        for (int i = 0; from[i]; ++i) t[(uint8_t)from[i]] = (uint8_t)to[i];
    }
};

uint8_t complement(uint8_t c) {
    static const ComplementTable table;  // initialised once, thread-safe
    return table.t[c];
}

int build(const char* data, int64_t n, int format, int64_t start, int64_t end, int64_t limit_length,
          int transform, int sort_desc, pw_records** out, char* err, int32_t err_bytes) {
    if (!out) return report(err, err_bytes, PW_ERR_ARG, "no output handle");
    *out = nullptr;
    if (n < 0 || (n > 0 && !data)) return report(err, err_bytes, PW_ERR_ARG, "bad input buffer");
    // islice(records, start, end): an end before the start selects nothing
    if (start < 0) return report(err, err_bytes, PW_ERR_ARG, "bad record range start %lld", (long long)start);
    if (transform < PW_RECORDS_AS_READ || transform > PW_RECORDS_APPEND_REVERSED)
        return report(err, err_bytes, PW_ERR_ARG, "unknown record transform %d", transform);
    std::vector<Rec> recs;
    std::vector<std::vector<uint8_t>> bufs;
    int rc;
    if (format == PW_FORMAT_FASTA) {
        rc = parse_fasta(data, n, recs, bufs);
    } else if (format == PW_FORMAT_FASTQ) {
        bufs.resize(1);
        rc = parse_fastq(data, n, recs, bufs[0], err, err_bytes);
        for (Rec& r : recs) r.s = bufs[0].data() + r.seq_begin;
    } else {
        return report(err, err_bytes, PW_ERR_ARG, "unknown record format %d", format);
    }
    if (rc != PW_OK) return rc;
    // islice(records, start, end)
    const int64_t total = (int64_t)recs.size();
    const int64_t r0 = std::min(start, total), r1 = end < 0 ? total : std::max(r0, std::min(end, total));
    pw_records* R = new pw_records();
    std::vector<int64_t> keep;
    keep.reserve((size_t)(r1 - r0));
    for (int64_t k = r0; k < r1; ++k) {
        const int64_t len = recs[k].seq_len;
        if (limit_length > 0 && (len > limit_length || len <= 0)) {
            R->dropped++;
            continue;
        }
        keep.push_back(k);
    }
    // the kept records, then their transformed copies
    const bool extra = transform != PW_RECORDS_AS_READ;
    const int64_t nk = (int64_t)keep.size();
    const int64_t nout = (transform == PW_RECORDS_APPEND_RC || transform == PW_RECORDS_APPEND_REVERSED) ? 2 * nk : nk;
    std::vector<int64_t> src(nout), lens(nout);
    std::vector<uint8_t> kind(nout);
    for (int64_t i = 0; i < nk; ++i) {
        if (transform == PW_RECORDS_RC_ONLY) {
            src[i] = keep[i];
            kind[i] = 1;
        } else {
            src[i] = keep[i];
            kind[i] = 0;
            if (extra) {
                src[nk + i] = keep[i];
                kind[nk + i] = transform == PW_RECORDS_APPEND_RC ? 1 : 2;
            }
        }
    }
    int64_t max_len = 0;
    for (int64_t i = 0; i < nout; ++i) {
        lens[i] = recs[src[i]].seq_len;
        max_len = std::max(max_len, lens[i]);
    }
    // a stable sort by length, longest first: ascending (max_len - length)
    std::vector<uint32_t> order;
    if (sort_desc) {
        std::vector<uint64_t> key((size_t)nout);
        for (int64_t i = 0; i < nout; ++i) key[i] = (uint64_t)(max_len - lens[i]);
        order = radix_order(std::move(key));
    } else {
        order.resize((size_t)nout);
        std::iota(order.begin(), order.end(), 0u);
    }
    R->src.resize((size_t)nout);
    R->kind.resize((size_t)nout);
    R->off.resize((size_t)nout + 1);
    R->id_off.resize((size_t)nout + 1);
    int64_t p = 0, q = 0;
    for (int64_t j = 0; j < nout; ++j) {
        const int64_t i = order[j];
        R->src[j] = src[i];
        R->kind[j] = kind[i];
        R->off[j] = p;
        R->id_off[j] = q;
        p += lens[i];
        q += recs[src[i]].id_len + (kind[i] ? 3 : 0);
    }
    R->off[nout] = p;
    R->id_off[nout] = q;
    R->ids.resize((size_t)q);
    parallel_for(nout, [&](int64_t j0, int64_t j1) {
        for (int64_t j = j0; j < j1; ++j) {
            const Rec& r = recs[R->src[j]];
            char* di = R->ids.data() + R->id_off[j];
            memcpy(di, data + r.id_begin, (size_t)r.id_len);
            if (R->kind[j]) memcpy(di + r.id_len, "_RC", 3);
        }
    }, 1 << 15);
    R->recs.swap(recs);
    R->bufs.swap(bufs);
    *out = R;
    return PW_OK;
}

}  // namespace

extern "C" int pw_records_parse(const char* data, int64_t bytes, int format, int64_t start, int64_t end,
                                int64_t limit_length, int transform, int sort_desc, pw_records** out, char* err,
                                int32_t err_bytes) {
    if (err && err_bytes > 0) err[0] = 0;
    return build(data, bytes, format, start, end, limit_length, transform, sort_desc, out, err, err_bytes);
}

extern "C" int pw_records_read(const char* path, int format, int64_t start, int64_t end, int64_t limit_length,
                               int transform, int sort_desc, pw_records** out, char* err, int32_t err_bytes) {
    if (err && err_bytes > 0) err[0] = 0;
    if (!path || !out) return report(err, err_bytes, PW_ERR_ARG, "no path or output handle");
    FILE* f = fopen(path, "rb");
    if (!f) return report(err, err_bytes, PW_ERR_ARG, "%s is not a file or cannot be read", path);
    std::string buf;
    char tmp[1 << 16];
    size_t got;
    while ((got = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, got);
    const bool bad = ferror(f) != 0;
    fclose(f);
    if (bad) return report(err, err_bytes, PW_ERR_ARG, "error reading %s", path);
    return build(buf.data(), (int64_t)buf.size(), format, start, end, limit_length, transform, sort_desc, out, err,
                 err_bytes);
}

extern "C" int pw_records_sizes(const pw_records* r, int64_t* n_records, int64_t* residue_bytes, int64_t* id_bytes,
                                int64_t* dropped) {
    if (!r) return PW_ERR_ARG;
    if (n_records) *n_records = (int64_t)r->off.size() - 1;
    if (residue_bytes) *residue_bytes = r->off.back();
    if (id_bytes) *id_bytes = (int64_t)r->ids.size();
    if (dropped) *dropped = r->dropped;
    return PW_OK;
}

extern "C" int pw_records_copy(const pw_records* r, uint8_t* residues, int64_t* offsets, char* ids,
                               int64_t* id_offsets) {
    if (!r) return PW_ERR_ARG;
    const int64_t n = (int64_t)r->src.size();
    if (residues)
        parallel_for(n, [&](int64_t j0, int64_t j1) {
            // SWSeqRecord upper-cases; the complement of an upper-case residue is upper case
            auto upper = [](uint8_t v) { return (v >= 'a' && v <= 'z') ? (uint8_t)(v - 32) : v; };
            for (int64_t j = j0; j < j1; ++j) {
                const Rec& rc = r->recs[r->src[j]];
                const uint8_t* s = rc.s;
                const int64_t L = rc.seq_len;
                uint8_t* d = residues + r->off[j];
                if (r->kind[j] == 0) {
                    for (int64_t k = 0; k < L; ++k) d[k] = upper(s[k]);
                } else if (r->kind[j] == 1) {
                    for (int64_t k = 0; k < L; ++k) d[k] = upper(complement(s[L - 1 - k]));
                } else {
                    for (int64_t k = 0; k < L; ++k) d[k] = upper(s[L - 1 - k]);
                }
            }
        }, 1 << 14);
    if (offsets) memcpy(offsets, r->off.data(), r->off.size() * sizeof(int64_t));
    if (ids && !r->ids.empty()) memcpy(ids, r->ids.data(), r->ids.size());
    if (id_offsets) memcpy(id_offsets, r->id_off.data(), r->id_off.size() * sizeof(int64_t));
    return PW_OK;
}

extern "C" void pw_records_free(pw_records* r) { delete r; }

// Dense ranks of n byte strings blob[off[i], off[i + 1]) in byte order, a
// string before every longer string it prefixes: the order of Python's str
// comparison on ASCII text (code points).  Equal strings share a rank.
// Sorted in pieces on host threads, then merged pairwise.
extern "C" int pw_id_ranks(const char* blob, const int64_t* off, int64_t n, int32_t* ranks) {
    if (n < 0 || (n > 0 && (!off || !ranks))) return PW_ERR_ARG;
    if (n == 0) return PW_OK;
    if (n > (int64_t)INT32_MAX) return PW_ERR_ARG;
    auto less = [&](uint32_t a, uint32_t b) {
        const int64_t la = off[a + 1] - off[a], lb = off[b + 1] - off[b];
        const int c = memcmp(blob + off[a], blob + off[b], (size_t)std::min(la, lb));
        return c < 0 || (c == 0 && la < lb);
    };
    std::vector<uint32_t> idx((size_t)n), tmp((size_t)n);
    std::iota(idx.begin(), idx.end(), 0u);
    const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    const int64_t pieces = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(hw, 32), n >> 14));
    std::vector<int64_t> cut((size_t)pieces + 1);
    for (int64_t k = 0; k <= pieces; ++k) cut[k] = n * k / pieces;
    parallel_for(pieces, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) std::sort(idx.begin() + cut[k], idx.begin() + cut[k + 1], less);
    }, 1);
    for (int64_t width = 1; width < pieces; width *= 2) {
        const int64_t merges = (pieces + 2 * width - 1) / (2 * width);
        parallel_for(merges, [&](int64_t m0, int64_t m1) {
            for (int64_t m = m0; m < m1; ++m) {
                const int64_t a = cut[m * 2 * width], b = cut[std::min(pieces, m * 2 * width + width)],
                              c = cut[std::min(pieces, m * 2 * width + 2 * width)];
                std::merge(idx.begin() + a, idx.begin() + b, idx.begin() + b, idx.begin() + c, tmp.begin() + a, less);
            }
        }, 1);
        idx.swap(tmp);
    }
    int32_t r = 0;
    for (int64_t k = 0; k < n; ++k) {
        if (k > 0 && less(idx[k - 1], idx[k])) ++r;
        ranks[idx[k]] = r;
    }
    return PW_OK;
}
