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
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/paswas_b200.h"

struct pw_records {
    std::vector<uint8_t> res;
    std::vector<int64_t> off;
    std::vector<char> ids;
    std::vector<int64_t> id_off;
    int64_t dropped = 0;  // records removed by the length limit
};

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

// One record as parsed: title id span in the input, sequence in `seq`.
struct Rec {
    int64_t id_begin, id_len;
    int64_t seq_begin, seq_len;  // in the parser's sequence buffer
};

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

int parse_fasta(const char* data, int64_t n, std::vector<Rec>& recs, std::vector<uint8_t>& seq) {
    Lines L{data, data + n};
    seq.reserve((size_t)n);
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
    std::vector<uint8_t> seq;
    int rc;
    if (format == PW_FORMAT_FASTA)
        rc = parse_fasta(data, n, recs, seq);
    else if (format == PW_FORMAT_FASTQ)
        rc = parse_fastq(data, n, recs, seq, err, err_bytes);
    else
        return report(err, err_bytes, PW_ERR_ARG, "unknown record format %d", format);
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
    std::vector<int> kind(nout);  // 0 as read, 1 reverse complement, 2 reversed
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
    for (int64_t i = 0; i < nout; ++i) lens[i] = recs[src[i]].seq_len;
    std::vector<int64_t> order(nout);
    std::iota(order.begin(), order.end(), 0);
    if (sort_desc) std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return lens[a] > lens[b]; });
    int64_t res_total = 0, id_total = 0;
    for (int64_t i = 0; i < nout; ++i) {
        res_total += lens[i];
        id_total += recs[src[i]].id_len + (kind[i] ? 3 : 0);
    }
    R->res.resize((size_t)res_total);
    R->off.resize((size_t)nout + 1);
    R->ids.resize((size_t)id_total);
    R->id_off.resize((size_t)nout + 1);
    int64_t p = 0, q = 0;
    for (int64_t j = 0; j < nout; ++j) {
        const int64_t i = order[j];
        const Rec& r = recs[src[i]];
        R->off[j] = p;
        const uint8_t* s = seq.data() + r.seq_begin;
        uint8_t* d = R->res.data() + p;
        // SWSeqRecord upper-cases; the complement of an upper-case residue is upper case
        auto upper = [](uint8_t v) { return (v >= 'a' && v <= 'z') ? (uint8_t)(v - 32) : v; };
        if (kind[i] == 0) {
            for (int64_t k = 0; k < r.seq_len; ++k) d[k] = upper(s[k]);
        } else if (kind[i] == 1) {
            for (int64_t k = 0; k < r.seq_len; ++k) d[k] = upper(complement(s[r.seq_len - 1 - k]));
        } else {
            for (int64_t k = 0; k < r.seq_len; ++k) d[k] = upper(s[r.seq_len - 1 - k]);
        }
        p += r.seq_len;
        R->id_off[j] = q;
        memcpy(R->ids.data() + q, data + r.id_begin, (size_t)r.id_len);
        q += r.id_len;
        if (kind[i]) {
            memcpy(R->ids.data() + q, "_RC", 3);
            q += 3;
        }
    }
    R->off[nout] = p;
    R->id_off[nout] = q;
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
    if (residue_bytes) *residue_bytes = (int64_t)r->res.size();
    if (id_bytes) *id_bytes = (int64_t)r->ids.size();
    if (dropped) *dropped = r->dropped;
    return PW_OK;
}

extern "C" int pw_records_copy(const pw_records* r, uint8_t* residues, int64_t* offsets, char* ids,
                               int64_t* id_offsets) {
    if (!r) return PW_ERR_ARG;
    if (residues && !r->res.empty()) memcpy(residues, r->res.data(), r->res.size());
    if (offsets) memcpy(offsets, r->off.data(), r->off.size() * sizeof(int64_t));
    if (ids && !r->ids.empty()) memcpy(ids, r->ids.data(), r->ids.size());
    if (id_offsets) memcpy(id_offsets, r->id_off.data(), r->id_off.size() * sizeof(int64_t));
    return PW_OK;
}

extern "C" void pw_records_free(pw_records* r) { delete r; }
