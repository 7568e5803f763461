/* hitbuild.c -- the driver's Hit / HitList construction in native code.
 *
 * SmithWatermanB200.align_sequences turns the engine's hit records (pw_hit,
 * include/paswas_b200.h) into the reference's Python objects: one Hit per
 * record that passes SmithWaterman._filter_hit (pyPaSWAS/Core/SmithWaterman.py
 * :843-848), with the attributes Hit.__init__ / set_scores give it
 * (pyPaSWAS/Core/Hit.py:16-119), appended to a HitList under its
 * start/end-key replacement rule (pyPaSWAS/Core/HitList.py:28-52).  This module
 * does exactly that for a whole record array in one call, so the per-hit work
 * runs in C instead of the interpreter; the objects it builds are the ones the
 * Python path builds (same attribute values, same dict entries, same order).
 *
 * build(hits, strbuf, sequences, targets, q_ids, t_ids, q_len, t_len, q_pos,
 *       t_pos, thresholds, hit_type, logger, hits_dict, real_dict)
 *   hits        buffer of pw_hit records (48 bytes each)
 *   strbuf      a bytes-like buffer: the alignment strings, n_cols bytes each at str_offset
 *   sequences, targets   the record lists the hit indices refer to
 *   q_ids, t_ids         lists of their ids
 *   q_len, t_len         buffers of int64 original lengths
 *   q_pos, t_pos         buffers of int64 start positions
 *   thresholds  (relative_score, query_identity, query_coverage, base_score)
 *   hit_type    the Hit class (instances get their attributes set directly)
 *   logger      the Hit's logger attribute
 *   hits_dict, real_dict  HitList.hits / HitList.real_hits, updated in place
 * Returns the number of hits kept by the filter, or None without touching the
 * dicts when a location is invalid (the caller then builds the hits through
 * the validating constructor, which raises at the first invalid one).
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    int32_t query, target, s_start, s_end, t_start, t_end;
    float score;
    int32_t matches, mismatches, n_cols;
    int64_t str_offset;
} HitRec;

enum {
    K_LOGGER, K_SEQ_INFO, K_TGT_INFO, K_SEQ_LOC, K_TGT_LOC, K_SEQ_MATCH, K_ALIGNMENT, K_TGT_MATCH, K_SCORE,
    K_MATCHES, K_MISMATCHES, K_IDENTITY, K_COVERAGE, K_RELATIVE, K_BASE, K_DISTANCE, K_RC, K_COUNT
};
static const char* kKeyNames[K_COUNT] = {
    "logger", "sequence_info", "target_info", "seq_location", "target_location", "sequence_match", "alignment",
    "target_match", "score", "matches", "mismatches", "query_identity", "query_coverage", "relative_score",
    "base_score", "distance", "rc"};
static PyObject* kKeys[K_COUNT];
static PyObject* kStrDistance;
static PyObject* kStrKeys;
static PyObject* kEmpty; /* () */

static int get_i64(Py_buffer* b, Py_ssize_t n, const char* what) {
    if (b->len != n * (Py_ssize_t)sizeof(int64_t)) {
        PyErr_Format(PyExc_ValueError, "%s: expected %zd int64 values", what, n);
        return -1;
    }
    return 0;
}

static PyObject* pair_of(int64_t a, int64_t b) {
    PyObject* t = PyTuple_New(2);
    if (!t) return NULL;
    PyObject* x = PyLong_FromLongLong(a);
    PyObject* y = PyLong_FromLongLong(b);
    if (!x || !y) {
        Py_XDECREF(x);
        Py_XDECREF(y);
        Py_DECREF(t);
        return NULL;
    }
    PyTuple_SET_ITEM(t, 0, x);
    PyTuple_SET_ITEM(t, 1, y);
    return t;
}

/* A tuple of exact str / int / float items cannot be part of a reference
 * cycle; the cyclic collector untracks such tuples on its first pass over
 * them.  Untracking them here, when they are made, spares that pass over the
 * four tuples of every hit. */
static void untrack_atoms(PyObject* t) {
    const Py_ssize_t n = PyTuple_GET_SIZE(t);
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* x = PyTuple_GET_ITEM(t, i);
        if (!(PyUnicode_CheckExact(x) || PyLong_CheckExact(x) || PyFloat_CheckExact(x))) return;
    }
    if (PyObject_GC_IsTracked(t)) PyObject_GC_UnTrack(t);
}

/* HitList.append's replacement rule for a new hit h with score sc and keys
 * k0 (start) / k1 (end) (HitList.py:28-52). */
static int hitlist_append(PyObject* hits_d, PyObject* real_d, PyObject* h, PyObject* sc, PyObject* k0,
                          PyObject* k1) {
    PyObject* old0 = PyDict_GetItemWithError(hits_d, k0); /* borrowed */
    if (!old0 && PyErr_Occurred()) return -1;
    PyObject* old1 = PyDict_GetItemWithError(hits_d, k1);
    if (!old1 && PyErr_Occurred()) return -1;
    int better_end = 0, better_start = 0;
    if (old1) {
        PyObject* s1 = PyObject_GetAttr(old1, kKeys[K_SCORE]);
        if (!s1) return -1;
        better_end = PyObject_RichCompareBool(s1, sc, Py_LT);
        Py_DECREF(s1);
        if (better_end < 0) return -1;
    }
    if (old0) {
        PyObject* s0 = PyObject_GetAttr(old0, kKeys[K_SCORE]);
        if (!s0) return -1;
        better_start = PyObject_RichCompareBool(s0, sc, Py_LT);
        Py_DECREF(s0);
        if (better_start < 0) return -1;
    }
    if (!((old0 == NULL && old1 == NULL) || better_end || better_start)) return 0;
    if (better_end) {
        /* the replaced hit's start key leaves real_hits (old1.keys()[2]) */
        Py_INCREF(old1);
        PyObject* ks = PyObject_CallMethodNoArgs(old1, kStrKeys);
        Py_DECREF(old1);
        if (!ks) return -1;
        PyObject* ok = PySequence_GetItem(ks, 2);
        Py_DECREF(ks);
        if (!ok) return -1;
        int has = PyDict_Contains(real_d, ok);
        if (has < 0 || (has && PyDict_DelItem(real_d, ok) < 0)) {
            Py_DECREF(ok);
            return -1;
        }
        Py_DECREF(ok);
    }
    if (PyDict_SetItem(hits_d, k0, h) < 0 || PyDict_SetItem(hits_d, k1, h) < 0 || PyDict_SetItem(real_d, k0, h) < 0)
        return -1;
    return 0;
}

static PyObject* build(PyObject* self, PyObject* args) {
    PyObject *hits_obj, *strbuf, *seqs, *tgts, *q_ids, *t_ids, *qlen_obj, *tlen_obj, *qpos_obj, *tpos_obj;
    PyObject *thr, *hit_type, *logger, *hits_d, *real_d;
    (void)self;
    if (!PyArg_ParseTuple(args, "OOO!O!O!O!OOOOOOOO!O!", &hits_obj, &strbuf, &PyList_Type, &seqs, &PyList_Type,
                          &tgts, &PyList_Type, &q_ids, &PyList_Type, &t_ids, &qlen_obj, &tlen_obj, &qpos_obj,
                          &tpos_obj, &thr, &hit_type, &logger, &PyDict_Type, &hits_d, &PyDict_Type, &real_d))
        return NULL;
    if (!PyType_Check(hit_type)) {
        PyErr_SetString(PyExc_TypeError, "hit_type must be a class");
        return NULL;
    }
    double th[4];
    if (!PyArg_ParseTuple(thr, "dddd", &th[0], &th[1], &th[2], &th[3])) return NULL;
    const Py_ssize_t nq = PyList_GET_SIZE(seqs), nt = PyList_GET_SIZE(tgts);
    if (PyList_GET_SIZE(q_ids) != nq || PyList_GET_SIZE(t_ids) != nt) {
        PyErr_SetString(PyExc_ValueError, "id lists do not match the record lists");
        return NULL;
    }
    Py_buffer hb, qlb, tlb, qpb, tpb, sb;
    if (PyObject_GetBuffer(strbuf, &sb, PyBUF_SIMPLE) < 0) return NULL;
    if (PyObject_GetBuffer(hits_obj, &hb, PyBUF_C_CONTIGUOUS) < 0) {
        PyBuffer_Release(&sb);
        return NULL;
    }
    int have[4] = {0, 0, 0, 0};
    int gc_was_on = 0;
    PyObject* result = NULL;
    if (PyObject_GetBuffer(qlen_obj, &qlb, PyBUF_C_CONTIGUOUS) < 0) goto done;
    have[0] = 1;
    if (PyObject_GetBuffer(tlen_obj, &tlb, PyBUF_C_CONTIGUOUS) < 0) goto done;
    have[1] = 1;
    if (PyObject_GetBuffer(qpos_obj, &qpb, PyBUF_C_CONTIGUOUS) < 0) goto done;
    have[2] = 1;
    if (PyObject_GetBuffer(tpos_obj, &tpb, PyBUF_C_CONTIGUOUS) < 0) goto done;
    have[3] = 1;
    if (hb.len % (Py_ssize_t)sizeof(HitRec) != 0) {
        PyErr_SetString(PyExc_ValueError, "hits: not a whole number of pw_hit records");
        goto done;
    }
    if (get_i64(&qlb, nq, "q_len") || get_i64(&tlb, nt, "t_len") || get_i64(&qpb, nq, "q_pos") ||
        get_i64(&tpb, nt, "t_pos"))
        goto done;
    {
        const HitRec* H = (const HitRec*)hb.buf;
        const Py_ssize_t n = hb.len / (Py_ssize_t)sizeof(HitRec);
        const int64_t *ql = (const int64_t*)qlb.buf, *tl = (const int64_t*)tlb.buf;
        const int64_t *qp = (const int64_t*)qpb.buf, *tp = (const int64_t*)tpb.buf;
        const char* text = (const char*)sb.buf;
        const Py_ssize_t text_len = sb.len;
        /* every location valid (Hit._is_a_valid_location), else the caller's path */
        for (Py_ssize_t k = 0; k < n; ++k) {
            const HitRec* r = &H[k];
            if (r->query < 0 || r->query >= nq || r->target < 0 || r->target >= nt || r->n_cols < 0 ||
                r->str_offset < 0 || r->str_offset + 3 * (int64_t)r->n_cols > (int64_t)text_len) {
                PyErr_SetString(PyExc_ValueError, "hit record outside the record lists or the string buffer");
                goto done;
            }
            const int64_t s0 = r->s_start + qp[r->query], s1 = r->s_end + qp[r->query];
            const int64_t t0 = r->t_start + tp[r->target], t1 = r->t_end + tp[r->target];
            if (!(0 <= s0 && s0 < s1 && s1 < ql[r->query] && 0 <= t0 && t0 < t1 && t1 < tl[r->target])) {
                result = Py_None;
                Py_INCREF(result);
                goto done;
            }
        }
        Py_ssize_t kept = 0;
        /* thousands of new container objects, none of them in a cycle: the
           cyclic collector is paused while they are made (restored below) */
        gc_was_on = PyGC_Disable();
        for (Py_ssize_t k = 0; k < n; ++k) {
            const HitRec* r = &H[k];
            const int64_t s0 = r->s_start + qp[r->query], s1 = r->s_end + qp[r->query];
            const int64_t t0 = r->t_start + tp[r->target], t1 = r->t_end + tp[r->target];
            const int64_t lq = ql[r->query], lt = tl[r->target];
            const double sc = (double)r->score;
            const double span = (double)(s1 - s0 + 1);
            /* the ratios of Hit.set_scores (Hit.py:108-119), IEEE double as Python's floats */
            const double rel = sc / (double)(lq > lt ? lt : lq);
            const double ident = (double)r->matches / span;
            const double cov = span / (double)lq;
            const double base = sc / (double)r->n_cols;
            if (!(rel >= th[0] && ident >= th[1] && cov >= th[2] && base >= th[3])) continue;
            PyObject* seq_rec = PyList_GET_ITEM(seqs, r->query); /* borrowed */
            PyObject* tgt_rec = PyList_GET_ITEM(tgts, r->target);
            /* SmithWaterman.py:743-744: records without a distance get 0.0 */
            if (!PyObject_HasAttr(seq_rec, kStrDistance)) {
                PyObject* z = PyFloat_FromDouble(0.0);
                if (!z || PyObject_SetAttr(seq_rec, kStrDistance, z) < 0) {
                    Py_XDECREF(z);
                    goto done;
                }
                Py_DECREF(z);
            }
            PyObject* v[K_COUNT];
            memset(v, 0, sizeof(v));
            const char* base_ptr = text + r->str_offset;
            v[K_LOGGER] = logger;
            Py_INCREF(logger);
            v[K_SEQ_INFO] = seq_rec;
            Py_INCREF(seq_rec);
            v[K_TGT_INFO] = tgt_rec;
            Py_INCREF(tgt_rec);
            v[K_SEQ_LOC] = pair_of(s0, s1);
            v[K_TGT_LOC] = pair_of(t0, t1);
            v[K_SEQ_MATCH] = PyUnicode_DecodeLatin1(base_ptr, r->n_cols, NULL);
            v[K_ALIGNMENT] = PyUnicode_DecodeLatin1(base_ptr + r->n_cols, r->n_cols, NULL);
            v[K_TGT_MATCH] = PyUnicode_DecodeLatin1(base_ptr + 2 * (int64_t)r->n_cols, r->n_cols, NULL);
            v[K_SCORE] = PyFloat_FromDouble(sc);
            v[K_MATCHES] = PyLong_FromLong(r->matches);
            v[K_MISMATCHES] = PyLong_FromLong(r->mismatches);
            v[K_IDENTITY] = PyFloat_FromDouble(ident);
            v[K_COVERAGE] = PyFloat_FromDouble(cov);
            v[K_RELATIVE] = PyFloat_FromDouble(rel);
            v[K_BASE] = PyFloat_FromDouble(base);
            v[K_DISTANCE] = Py_None;
            Py_INCREF(Py_None);
            v[K_RC] = Py_False;
            Py_INCREF(Py_False);
            PyObject *h = NULL, *k0 = NULL, *k1 = NULL, *a0 = NULL, *b0 = NULL, *a1 = NULL, *b1 = NULL;
            int ok = 1;
            for (int i = 0; i < K_COUNT; ++i)
                if (!v[i]) ok = 0;
            if (ok) {
                /* the class's __new__ (object_new) readies the instance's
                   inline attribute values; the attributes follow in
                   Hit.__init__'s order (the class's shared key order) */
                h = ((PyTypeObject*)hit_type)->tp_new((PyTypeObject*)hit_type, kEmpty, NULL);
                ok = h != NULL;
                for (int i = 0; ok && i < K_COUNT; ++i) ok = PyObject_GenericSetAttr(h, kKeys[i], v[i]) == 0;
            }
            if (ok) {
                /* HitList keys (Hit.keys, Hit.py:151-158): start, end */
                PyObject* qid = PyList_GET_ITEM(q_ids, r->query);
                PyObject* tid = PyList_GET_ITEM(t_ids, r->target);
                a0 = PyTuple_GET_ITEM(v[K_SEQ_LOC], 0);
                a1 = PyTuple_GET_ITEM(v[K_SEQ_LOC], 1);
                b0 = PyTuple_GET_ITEM(v[K_TGT_LOC], 0);
                b1 = PyTuple_GET_ITEM(v[K_TGT_LOC], 1);
                k0 = PyTuple_Pack(4, qid, tid, a0, b0);
                k1 = PyTuple_Pack(4, qid, tid, a1, b1);
                untrack_atoms(v[K_SEQ_LOC]);
                untrack_atoms(v[K_TGT_LOC]);
                if (k0) untrack_atoms(k0);
                if (k1) untrack_atoms(k1);
                ok = k0 && k1 && hitlist_append(hits_d, real_d, h, v[K_SCORE], k0, k1) == 0;
            }
            Py_XDECREF(k0);
            Py_XDECREF(k1);
            Py_XDECREF(h);
            for (int i = 0; i < K_COUNT; ++i) Py_XDECREF(v[i]);
            if (!ok) goto done;
            ++kept;
        }
        result = PyLong_FromSsize_t(kept);
    }
done:
    if (gc_was_on) PyGC_Enable();
    PyBuffer_Release(&sb);
    PyBuffer_Release(&hb);
    if (have[0]) PyBuffer_Release(&qlb);
    if (have[1]) PyBuffer_Release(&tlb);
    if (have[2]) PyBuffer_Release(&qpb);
    if (have[3]) PyBuffer_Release(&tpb);
    return result;
}

static PyMethodDef kMethods[] = {
    {"build", build, METH_VARARGS, "Hit objects of engine hit records, appended to a HitList's dicts."},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_hitbuild", NULL, -1, kMethods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__hitbuild(void) {
    for (int i = 0; i < K_COUNT; ++i) {
        kKeys[i] = PyUnicode_InternFromString(kKeyNames[i]);
        if (!kKeys[i]) return NULL;
    }
    kStrDistance = PyUnicode_InternFromString("distance");
    kStrKeys = PyUnicode_InternFromString("keys");
    kEmpty = PyTuple_New(0);
    if (!kEmpty) return NULL;
    if (!kStrDistance || !kStrKeys) return NULL;
    return PyModule_Create(&kModule);
}
