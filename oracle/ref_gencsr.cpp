// ORACLE — test infrastructure only, never shipped or linked by the engine.
//
// Exposes the reference's own Python-graph -> C++ graph conversion and its
// out-edge CSR builder as a small Python module (_ref_gencsr), so the tests can
// check the engine's graph walk array for array against them:
//   build_graph / build_digraph   cpp_easygraph/classes/graph_convert.cpp:72-134
//   Graph::gen_CSR()              cpp_easygraph/classes/graph.cpp:819-886
//   Graph::gen_CSR(weight)        cpp_easygraph/classes/graph.cpp:719-817
// The reference's conversion functions live in an anonymous namespace of
// graph_convert.cpp, so this translation unit #includes that file from the
// reference tree (include path from oracle/Makefile.gencsr); nothing is copied.
#include "classes/graph_convert.cpp"

#include <pybind11/numpy.h>

namespace {

template <typename T>
py::array_t<T> to_array(const std::vector<T>& v) {
    py::array_t<T> a((py::ssize_t)v.size());
    if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), v.size() * sizeof(T));
    return a;
}

py::tuple csr_of(Graph& g, const py::object& weight) {
    std::shared_ptr<CSRGraph> c;
    py::object w = py::none();
    if (weight.is_none()) {
        c = g.gen_CSR();
    } else {
        const std::string key = weight.cast<std::string>();
        c = g.gen_CSR(key);
        w = to_array(*c->W_map[key]);
    }
    return py::make_tuple(to_array(c->V), to_array(c->E), w);
}

}  // namespace

PYBIND11_MODULE(_ref_gencsr, m) {
    m.doc() = "The reference's graph conversion and gen_CSR (oracle test infrastructure)";
    m.def(
        "gen_csr",
        [](py::object G, bool directed, py::object weight) {
            if (directed) {
                DiGraph d = build_digraph(G);
                return csr_of(d, weight);
            }
            Graph u = build_graph(G);
            return csr_of(u, weight);
        },
        py::arg("G"), py::arg("directed"), py::arg("weight") = py::none());
}
