// Python graph -> out-edge CSR in native code (CPython extension `_graph_walk`).
//
// Walks the adjacency dict of an EasyGraph graph ({u: {v: attr}}) once and
// builds V/E/W with the rules of build_digraph / build_graph
// (cpp_easygraph/classes/graph_convert.cpp:72-134) and gen_CSR
// (cpp_easygraph/classes/graph.cpp:719-886):
//   * rows in node-index order (the index dict maps node -> position);
//   * directed graphs keep every arc, self-loops included;
//   * undirected graphs drop self-loops and keep each unordered pair once per
//     direction, the pair's weight taken where it is first met;
//   * each row sorted by destination index;
//   * a weight is attr[weight] converted with float(), 1.0 when the attribute
//     is missing, the attribute dict is empty, or the conversion fails.
// The same walk in Python (eggpu_b200.backend._graph_csr_py) is the
// specification; tests compare the two array for array.
//
// out_csr(adj, index, n, directed, weight) -> (V, E, W) as bytearrays
// (int32 n+1, int32 m, float64 m or None), or None when adj / its rows are not
// plain dicts (the caller then walks in Python).
//
// stamp(adj) -> (nodes, adjacency slots, h): the prepared-graph fingerprint of
// backend._graph_stamp_py (node count, adjacency slots, a 64-bit mix of node
// hashes and degrees and of the first 4 neighbours of the first 32 nodes),
// value for value, or None when adj / its rows are not plain dicts.
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace {

// The unordered pairs {u, v} an undirected walk has met, keyed lo << 32 | hi
// (both below 2^31, so the all-ones word never is a key).  Open addressing
// with linear probing, sized up front to at least twice the adjacency's
// entries: one probe sequence per visit, no rehashing.
class PairSet {
public:
    explicit PairSet(size_t entries) {
        size_t cap = 16;
        while (cap < 2 * entries) cap <<= 1;
        slots_.assign(cap, kEmpty);
        mask_ = cap - 1;
    }
    // true when the pair was not in the set yet
    bool insert(uint64_t key) {
        for (uint64_t h = mix(key) & mask_;; h = (h + 1) & mask_) {
            const uint64_t s = slots_[h];
            if (s == key) return false;
            if (s == kEmpty) {
                slots_[h] = key;
                return true;
            }
        }
    }

private:
    static constexpr uint64_t kEmpty = ~0ull;
    static uint64_t mix(uint64_t x) {  // SplitMix64 finaliser
        x ^= x >> 30;
        x *= 0xbf58476d1ce4e5b9ull;
        x ^= x >> 27;
        x *= 0x94d049bb133111ebull;
        return x ^ (x >> 31);
    }
    std::vector<uint64_t> slots_;
    uint64_t mask_ = 0;
};

// float(attr.get(weight, 1.0)) with the fallbacks of backend._weight_of.
bool weight_of(PyObject* attr, PyObject* weight, double* out) {
    *out = 1.0;
    if (attr == nullptr || attr == Py_None) return true;
    const int truth = PyObject_IsTrue(attr);
    if (truth < 0) return false;
    if (truth == 0) return true;
    PyObject* val = nullptr;
    if (PyDict_Check(attr)) {
        val = PyDict_GetItemWithError(attr, weight);  // borrowed
        if (val == nullptr) return !PyErr_Occurred();
        Py_INCREF(val);
    } else {
        val = PyObject_CallMethod(attr, "get", "OO", weight, Py_None);
        if (val == nullptr) return false;
        if (val == Py_None) {
            Py_DECREF(val);
            return true;
        }
    }
    PyObject* f = PyNumber_Float(val);
    Py_DECREF(val);
    if (f == nullptr) {
        if (PyErr_ExceptionMatches(PyExc_TypeError) || PyErr_ExceptionMatches(PyExc_ValueError)) {
            PyErr_Clear();
            return true;
        }
        return false;
    }
    *out = PyFloat_AS_DOUBLE(f);
    Py_DECREF(f);
    return true;
}

bool index_of(PyObject* index, PyObject* node, int64_t n, int32_t* out) {
    PyObject* i = PyDict_GetItemWithError(index, node);  // borrowed
    if (i == nullptr) {
        if (!PyErr_Occurred()) PyErr_SetObject(PyExc_KeyError, node);
        return false;
    }
    const long long v = PyLong_AsLongLong(i);
    if (v == -1 && PyErr_Occurred()) return false;
    if (v < 0 || v >= n) {
        PyErr_SetString(PyExc_IndexError, "node index out of range");
        return false;
    }
    *out = (int32_t)v;
    return true;
}

PyObject* out_csr(PyObject*, PyObject* args) {
    PyObject *adj, *index, *weight;
    Py_ssize_t n;
    int directed;
    if (!PyArg_ParseTuple(args, "OOnpO", &adj, &index, &n, &directed, &weight)) return nullptr;
    if (!PyDict_Check(adj) || !PyDict_Check(index)) Py_RETURN_NONE;
    if (n < 0 || n >= INT32_MAX) {
        PyErr_SetString(PyExc_ValueError, "node count exceeds the signed 32-bit CSR limit");
        return nullptr;
    }
    const bool want_w = weight != Py_None;
    // first pass: every row a plain dict, and the adjacency's total size
    size_t entries = 0;
    {
        PyObject *u, *nbrs;
        Py_ssize_t pos = 0;
        while (PyDict_Next(adj, &pos, &u, &nbrs)) {
            if (!PyDict_Check(nbrs)) Py_RETURN_NONE;
            entries += (size_t)PyDict_Size(nbrs);
        }
    }
    std::vector<int32_t> src, dst;
    std::vector<double> wts;
    src.reserve(entries);
    dst.reserve(entries);
    if (want_w) wts.reserve(entries);
    PairSet seen(directed ? 0 : entries);
    {
        PyObject *u, *nbrs;
        Py_ssize_t pos = 0;
        while (PyDict_Next(adj, &pos, &u, &nbrs)) {
            if (!PyDict_Check(nbrs)) Py_RETURN_NONE;
            int32_t iu;
            if (!index_of(index, u, n, &iu)) return nullptr;
            PyObject *v, *attr;
            Py_ssize_t p2 = 0;
            while (PyDict_Next(nbrs, &p2, &v, &attr)) {
                int32_t iv;
                if (!index_of(index, v, n, &iv)) return nullptr;
                if (directed) {
                    double w = 1.0;
                    if (want_w && !weight_of(attr, weight, &w)) return nullptr;
                    src.push_back(iu);
                    dst.push_back(iv);
                    if (want_w) wts.push_back(w);
                } else {
                    if (iu == iv) continue;
                    const uint64_t key = iu < iv ? ((uint64_t)(uint32_t)iu << 32) | (uint32_t)iv
                                                 : ((uint64_t)(uint32_t)iv << 32) | (uint32_t)iu;
                    if (!seen.insert(key)) continue;
                    double w = 1.0;
                    if (want_w && !weight_of(attr, weight, &w)) return nullptr;
                    src.push_back(iu);
                    dst.push_back(iv);
                    src.push_back(iv);
                    dst.push_back(iu);
                    if (want_w) {
                        wts.push_back(w);
                        wts.push_back(w);
                    }
                }
            }
        }
    }
    const size_t m = src.size();
    if (m >= (size_t)INT32_MAX) {
        PyErr_SetString(PyExc_ValueError, "adjacency entry count exceeds the signed 32-bit CSR limit");
        return nullptr;
    }
    // counting sort by source, then each row by destination
    std::vector<int64_t> V((size_t)n + 1, 0);
    for (size_t i = 0; i < m; ++i) V[(size_t)src[i] + 1] += 1;
    for (Py_ssize_t r = 0; r < n; ++r) V[(size_t)r + 1] += V[(size_t)r];
    std::vector<int64_t> cur(V.begin(), V.end() - 1);
    std::vector<int32_t> E(std::max<size_t>(m, 1));
    std::vector<double> W(want_w ? std::max<size_t>(m, 1) : 0);
    std::vector<std::pair<int32_t, double>> row;
    {
        std::vector<int64_t> slot(m);
        for (size_t i = 0; i < m; ++i) slot[i] = cur[(size_t)src[i]]++;
        for (size_t i = 0; i < m; ++i) {
            E[(size_t)slot[i]] = dst[i];
            if (want_w) W[(size_t)slot[i]] = wts[i];
        }
    }
    for (Py_ssize_t r = 0; r < n; ++r) {
        const int64_t b = V[(size_t)r], e = V[(size_t)r + 1];
        if (e - b < 2) continue;
        if (!want_w) {
            std::sort(E.begin() + b, E.begin() + e);
        } else {
            row.clear();
            for (int64_t i = b; i < e; ++i) row.emplace_back(E[(size_t)i], W[(size_t)i]);
            std::sort(row.begin(), row.end(),
                      [](const std::pair<int32_t, double>& x, const std::pair<int32_t, double>& y) {
                          return x.first < y.first;
                      });
            for (int64_t i = b; i < e; ++i) {
                E[(size_t)i] = row[(size_t)(i - b)].first;
                W[(size_t)i] = row[(size_t)(i - b)].second;
            }
        }
    }
    std::vector<int32_t> V32((size_t)n + 1);
    for (size_t i = 0; i <= (size_t)n; ++i) V32[i] = (int32_t)V[i];
    PyObject* pv = PyByteArray_FromStringAndSize(reinterpret_cast<const char*>(V32.data()),
                                                 (Py_ssize_t)(V32.size() * sizeof(int32_t)));
    PyObject* pe = PyByteArray_FromStringAndSize(reinterpret_cast<const char*>(E.data()),
                                                 (Py_ssize_t)(m * sizeof(int32_t)));
    PyObject* pw = nullptr;
    if (want_w) {
        pw = PyByteArray_FromStringAndSize(reinterpret_cast<const char*>(W.data()), (Py_ssize_t)(m * sizeof(double)));
    } else {
        Py_INCREF(Py_None);
        pw = Py_None;
    }
    if (!pv || !pe || !pw) {
        Py_XDECREF(pv);
        Py_XDECREF(pe);
        Py_XDECREF(pw);
        return nullptr;
    }
    PyObject* out = PyTuple_Pack(3, pv, pe, pw);
    Py_DECREF(pv);
    Py_DECREF(pe);
    Py_DECREF(pw);
    return out;
}

// h ^= x + 0x9E3779B97F4A7C15 + (h << 6) + (h >> 2), all modulo 2^64
// (backend._mix64; x is a Python hash, taken in two's complement).
uint64_t mix64(uint64_t h, int64_t x) {
    return h ^ ((uint64_t)x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2));
}

PyObject* stamp(PyObject*, PyObject* args) {
    PyObject* adj;
    if (!PyArg_ParseTuple(args, "O", &adj)) return nullptr;
    if (!PyDict_Check(adj)) Py_RETURN_NONE;
    uint64_t h = 1469598103934665603ull;
    unsigned long long slots = 0;
    PyObject *u, *nbrs;
    Py_ssize_t pos = 0, i = 0;
    while (PyDict_Next(adj, &pos, &u, &nbrs)) {
        if (!PyDict_Check(nbrs)) Py_RETURN_NONE;
        const Py_ssize_t deg = PyDict_Size(nbrs);
        slots += (unsigned long long)deg;
        const Py_hash_t hu = PyObject_Hash(u);
        if (hu == -1 && PyErr_Occurred()) return nullptr;
        h = mix64(h, (int64_t)hu);
        h = mix64(h, (int64_t)deg);
        if (i < 32) {
            PyObject *v, *attr;
            Py_ssize_t p2 = 0;
            for (int j = 0; j < 4 && PyDict_Next(nbrs, &p2, &v, &attr); ++j) {
                const Py_hash_t hv = PyObject_Hash(v);
                if (hv == -1 && PyErr_Occurred()) return nullptr;
                h = mix64(h, (int64_t)hv);
            }
        }
        ++i;
    }
    return Py_BuildValue("(nKK)", PyDict_Size(adj), slots, (unsigned long long)h);
}

PyMethodDef kMethods[] = {
    {"out_csr", out_csr, METH_VARARGS,
     "out_csr(adj, index, n, directed, weight) -> (V, E, W) bytearrays, or None for non-dict adjacency"},
    {"stamp", stamp, METH_VARARGS, "stamp(adj) -> (nodes, adjacency slots, fingerprint), or None for non-dict adjacency"},
    {nullptr, nullptr, 0, nullptr},
};

PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_graph_walk", "Python graph -> out-edge CSR", -1, kMethods};

}  // namespace

PyMODINIT_FUNC PyInit__graph_walk(void) { return PyModule_Create(&kModule); }
