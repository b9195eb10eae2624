// ORACLE / TEST INFRASTRUCTURE ONLY. Never shipped, never on the product path.
//
// A project-written pybind11 module named `_native` that binds the reference's own, unmodified,
// header-only wave solver (cpp/include/acoustic_spaces/fdtd.hpp, bvh.hpp, cut_cells.hpp of
// naelolaiz/acoustic-spaces). The reference's own binding (cpp/bindings/native_module.cpp) needs
// nanobind, which this image lacks; this module exposes the same names, argument names and
// defaults for the parts the wave stage and its tests use:
//   Bvh(vertices, faces, split="sah")                     cpp/bindings/native_module.cpp:1422-1435
//   WaveSolver(bvh, face_material, beta, branches, ...)   cpp/bindings/native_module.cpp:1238-1283,
//                                                         1564-1707
//   CutFit(vertices, faces, face_material, materials, ...) cpp/bindings/native_module.cpp:1465-1559
// so that `acoustic_spaces._native` can be replaced by it under the reference's Python sources.
// Its compiled form lives in oracle/_ref/ (built by oracle/Makefile from the reference headers
// where they lie; no reference source is copied into this repository).

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cstdint>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "acoustic_spaces/bvh.hpp"
#include "acoustic_spaces/fdtd.hpp"

namespace py = pybind11;
namespace as = acoustic_spaces;

namespace {

template <typename T>
using CArray = py::array_t<T, py::array::c_style | py::array::forcecast>;

template <typename T>
py::array to_numpy(const std::vector<T> &values) {
    using Out = std::conditional_t<std::is_same_v<T, std::size_t>, std::uint64_t, T>;
    py::array_t<Out> out(static_cast<py::ssize_t>(values.size()));
    auto *dst = out.mutable_data();
    for (std::size_t i = 0; i < values.size(); ++i) dst[i] = static_cast<Out>(values[i]);
    return out;
}

std::vector<as::Vec3> points_of(const CArray<double> &a, const char *what) {
    if (a.ndim() == 1 && a.shape(0) == 0) return {};
    if (a.ndim() != 2 || a.shape(1) != 3) throw std::invalid_argument(std::string(what) + ": (n, 3)");
    std::vector<as::Vec3> out(static_cast<std::size_t>(a.shape(0)));
    const double *d = a.data();
    for (std::size_t i = 0; i < out.size(); ++i) out[i] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    return out;
}

as::Vec3 vec_of(const CArray<double> &a, const char *what) {
    if (a.size() != 3) throw std::invalid_argument(std::string(what) + " needs 3 values");
    return {a.data()[0], a.data()[1], a.data()[2]};
}

// The reference's tree together with copies of the arrays it was built from (the fitted path
// reads the mesh again while the solver is set up).
struct BvhHolder {
    std::vector<double> vertices;
    std::vector<std::int64_t> faces;
    std::unique_ptr<as::Bvh> bvh;
};

struct SolverHolder {
    std::unique_ptr<as::WaveSolver> solver;
};

std::shared_ptr<BvhHolder> make_bvh(const CArray<double> &vertices, const CArray<std::int64_t> &faces,
                                    const std::string &split) {
    if (split != "sah" && split != "median") throw std::invalid_argument("Bvh: split must be 'sah' or 'median'");
    if (vertices.ndim() != 2 || vertices.shape(1) != 3) throw std::invalid_argument("Bvh: vertices (n, 3)");
    if (faces.ndim() != 2 || faces.shape(1) != 3) throw std::invalid_argument("Bvh: faces (m, 3)");
    auto h = std::make_shared<BvhHolder>();
    h->vertices.assign(vertices.data(), vertices.data() + vertices.size());
    h->faces.assign(faces.data(), faces.data() + faces.size());
    h->bvh = std::make_unique<as::Bvh>(h->vertices.data(), static_cast<std::size_t>(vertices.shape(0)),
                                       h->faces.data(), static_cast<std::size_t>(faces.shape(0)),
                                       split == "sah" ? as::BvhSplit::kSah : as::BvhSplit::kMedian);
    return h;
}

std::shared_ptr<SolverHolder> make_solver(
    const BvhHolder &bvh, const CArray<std::int64_t> &face_material, const CArray<double> &beta,
    const CArray<double> &branches, const CArray<std::int64_t> &branch_material, const CArray<double> &origin,
    double cell, std::size_t nx, std::size_t ny, std::size_t nz, const CArray<double> &source,
    const CArray<double> &probes, double edge_admittance, std::size_t layer, double layer_damping,
    std::size_t threads, std::size_t stencil, std::optional<CArray<float>> speed,
    std::optional<CArray<float>> flow_x, std::optional<CArray<float>> flow_y, std::size_t probes_per_listener,
    bool fitted_walls, std::optional<CArray<double>> vertices, std::optional<CArray<std::int64_t>> faces) {
    if (static_cast<std::size_t>(face_material.size()) != bvh.bvh->face_count())
        throw std::invalid_argument("WaveSolver: one material per face");
    const std::size_t count = static_cast<std::size_t>(branch_material.size());
    if (count > 0 && (branches.ndim() != 2 || static_cast<std::size_t>(branches.shape(0)) != count ||
                      branches.shape(1) != 3))
        throw std::invalid_argument("WaveSolver: m, r and q of each branch, and its material");
    const std::size_t n = nx * ny * nz;
    if (speed && static_cast<std::size_t>(speed->size()) != n)
        throw std::invalid_argument("WaveSolver: one speed per cell of the grid");
    if (flow_x.has_value() != flow_y.has_value())
        throw std::invalid_argument("WaveSolver: flow_x and flow_y go together");
    if (flow_x && (static_cast<std::size_t>(flow_x->size()) != n || static_cast<std::size_t>(flow_y->size()) != n))
        throw std::invalid_argument("WaveSolver: one shift of the air per cell of the grid");
    const std::vector<as::Vec3> probe_points = points_of(probes, "probes");
    const as::Vec3 o = vec_of(origin, "origin"), s = vec_of(source, "source");
    as::CutCells::Mesh mesh;
    std::vector<double> vs;
    std::vector<std::int64_t> fs;
    if (fitted_walls) {
        if (!vertices || !faces)
            throw std::invalid_argument("fitted walls: the solver needs the vertices and faces the BVH was built from");
        vs.assign(vertices->data(), vertices->data() + vertices->size());
        fs.assign(faces->data(), faces->data() + faces->size());
        mesh.vertices = vs.data();
        mesh.vertex_count = vs.size() / 3;
        mesh.faces = fs.data();
        mesh.face_count = fs.size() / 3;
        for (std::size_t i = 0; i < fs.size(); ++i)
            if (fs[i] < 0 || static_cast<std::size_t>(fs[i]) >= mesh.vertex_count)
                throw std::invalid_argument("fitted walls: a face refers to a missing vertex");
        if (mesh.face_count != bvh.bvh->face_count())
            throw std::invalid_argument("fitted walls: the faces given are not the BVH's (their counts differ)");
    }
    auto h = std::make_shared<SolverHolder>();
    {
        py::gil_scoped_release release;
        h->solver = std::make_unique<as::WaveSolver>(
            *bvh.bvh, face_material.data(), beta.data(), static_cast<std::size_t>(beta.size()),
            count ? branches.data() : nullptr, branch_material.data(), count, o, cell, nx, ny, nz, s, probe_points,
            edge_admittance, layer, layer_damping, threads, stencil, speed ? speed->data() : nullptr,
            flow_x ? flow_x->data() : nullptr, flow_y ? flow_y->data() : nullptr, probes_per_listener,
            fitted_walls, fitted_walls ? &mesh : nullptr);
    }
    return h;
}

// The fit alone (the reference's CutCells on the wave solver's grid; its own binding is CutFit,
// cpp/bindings/native_module.cpp:1465-1559): the vertices and faces are kept for the fit's life.
struct FitHolder {
    std::vector<double> vertices;
    std::vector<std::int64_t> faces;
    std::unique_ptr<as::CutCells> cut;
};

std::shared_ptr<FitHolder> make_fit(const CArray<double> &vertices, const CArray<std::int64_t> &faces,
                                    const CArray<std::int64_t> &face_material, std::size_t materials,
                                    const CArray<double> &origin, double cell, std::size_t nx, std::size_t ny,
                                    std::size_t nz, const CArray<double> &source, std::size_t layer,
                                    std::size_t threads) {
    if (vertices.ndim() != 2 || vertices.shape(1) != 3) throw std::invalid_argument("CutFit: vertices (n, 3)");
    if (faces.ndim() != 2 || faces.shape(1) != 3) throw std::invalid_argument("CutFit: faces (m, 3)");
    if (face_material.size() != faces.shape(0)) throw std::invalid_argument("CutFit: one material per face");
    auto h = std::make_shared<FitHolder>();
    h->vertices.assign(vertices.data(), vertices.data() + vertices.size());
    h->faces.assign(faces.data(), faces.data() + faces.size());
    for (std::int64_t f : h->faces)
        if (f < 0 || static_cast<std::size_t>(f) >= h->vertices.size() / 3)
            throw std::invalid_argument("CutFit: a face refers to a missing vertex");
    for (py::ssize_t f = 0; f < face_material.size(); ++f)
        if (face_material.data()[f] < 0 || static_cast<std::size_t>(face_material.data()[f]) >= materials)
            throw std::invalid_argument("CutFit: a face's material is not below materials");
    as::CutCells::Mesh mesh;
    mesh.vertices = h->vertices.data();
    mesh.vertex_count = h->vertices.size() / 3;
    mesh.faces = h->faces.data();
    mesh.face_count = h->faces.size() / 3;
    const as::Vec3 o = vec_of(origin, "origin"), src = vec_of(source, "source");
    {
        py::gil_scoped_release release;
        h->cut = std::make_unique<as::CutCells>(mesh, face_material.data(), materials,
                                                as::WaveSolver::cut_grid(o, cell, nx, ny, nz, layer), src, threads);
    }
    if (h->cut->refused()) throw std::invalid_argument(h->cut->refusal());
    return h;
}

template <typename T>
py::array shaped(const std::vector<T> &values, std::size_t rows, std::size_t cols) {
    py::array_t<T> out({static_cast<py::ssize_t>(rows), static_cast<py::ssize_t>(cols)});
    std::copy(values.begin(), values.end(), out.mutable_data());
    return out;
}

py::dict fit_cells(const FitHolder &h) {
    const as::CutCells &cut = *h.cut;
    const std::size_t n = cut.cells().size(), w = cut.materials() + 1;
    py::dict out;
    out["cell"] = to_numpy(cut.cells());
    out["air_volume"] = to_numpy(cut.air_volume());
    out["open_area"] = shaped(cut.open_area(), n, 18);
    out["wall_area"] = shaped(cut.wall_area(), n, w);
    out["sliver"] = shaped(cut.sliver(), n, 6);
    return out;
}

py::array run(SolverHolder &h, const CArray<float> &signal) {
    if (signal.ndim() != 1) throw std::invalid_argument("run: the signal is 1-D");
    const std::size_t steps = static_cast<std::size_t>(signal.shape(0));
    const std::size_t probes = h.solver->probes();
    py::array_t<double> out({static_cast<py::ssize_t>(probes), static_cast<py::ssize_t>(steps)});
    double *dst = out.mutable_data();
    const float *src = signal.data();
    {
        py::gil_scoped_release release;
        h.solver->run(src, steps, dst);
    }
    return out;
}

py::dict layout(const SolverHolder &h) {
    py::dict out;
    h.solver->layout([&](const char *name, const auto &values) { out[name] = to_numpy(values); });
    return out;
}

}  // namespace

PYBIND11_MODULE(_native, m) {
    m.doc() = "The reference wave solver's unmodified C++ core, bound for use as a test oracle.";

    py::class_<BvhHolder, std::shared_ptr<BvhHolder>>(m, "Bvh")
        .def(py::init(&make_bvh), py::arg("vertices"), py::arg("faces"), py::arg("split") = "sah")
        .def_property_readonly("face_count", [](const BvhHolder &h) { return h.bvh->face_count(); })
        .def(
            "set_facing",
            [](BvhHolder &h, const CArray<std::int8_t> &facing) {
                if (static_cast<std::size_t>(facing.size()) != h.bvh->face_count())
                    throw std::invalid_argument("Bvh.set_facing: one value per face");
                h.bvh->set_facing(facing.data());
            },
            py::arg("facing"))
        .def_property_readonly("has_facing", [](const BvhHolder &h) { return h.bvh->has_facing(); });

    py::class_<SolverHolder, std::shared_ptr<SolverHolder>>(m, "WaveSolver")
        .def(py::init(&make_solver), py::arg("bvh"), py::arg("face_material"), py::arg("beta"), py::arg("branches"),
             py::arg("branch_material"), py::arg("origin"), py::arg("cell"), py::arg("nx"), py::arg("ny"),
             py::arg("nz"), py::arg("source"), py::arg("probes"), py::arg("edge_admittance") = 1.0,
             py::arg("layer") = 0, py::arg("layer_damping") = 0.0, py::arg("threads") = 0,
             py::arg("stencil") = 7, py::arg("speed") = py::none(), py::arg("flow_x") = py::none(),
             py::arg("flow_y") = py::none(), py::arg("probes_per_listener") = 1, py::arg("fitted_walls") = false,
             py::arg("vertices") = py::none(), py::arg("faces") = py::none())
        .def_property_readonly("air_cells", [](const SolverHolder &h) { return h.solver->air_cells(); })
        .def_property_readonly("boundary_cells", [](const SolverHolder &h) { return h.solver->boundary_cells(); })
        .def_property_readonly("branch_states", [](const SolverHolder &h) { return h.solver->branch_states(); })
        .def_property_readonly("layer_cells", [](const SolverHolder &h) { return h.solver->layer_cells(); })
        .def_property_readonly("open", [](const SolverHolder &h) { return h.solver->open(); })
        .def_property_readonly("open_sides",
                               [](const SolverHolder &h) {
                                   const auto &s = h.solver->open_sides();
                                   return py::make_tuple(s[0], s[1], s[2], s[3], s[4], s[5]);
                               })
        .def_property_readonly("flowing", [](const SolverHolder &h) { return h.solver->flowing(); })
        .def_property_readonly("wind_round", [](const SolverHolder &h) { return h.solver->wind_round(); })
        .def_property_readonly("wind_fastest", [](const SolverHolder &h) { return h.solver->wind_fastest(); })
        .def_property_readonly("wind_sweeps", [](const SolverHolder &h) { return h.solver->wind_sweeps(); })
        .def_property_readonly("mean_square", [](const SolverHolder &h) { return h.solver->mean_square(); })
        .def_property_readonly("stencil", [](const SolverHolder &h) { return h.solver->stencil(); })
        .def_property_readonly("threads", [](const SolverHolder &h) { return h.solver->threads(); })
        .def_property_readonly("fitted_walls", [](const SolverHolder &h) { return h.solver->cut_cells() != nullptr; })
        .def_property_readonly("cut_stats",
                               [](const SolverHolder &h) {
                                   py::dict d;
                                   const auto *cut = h.solver->cut_cells();
                                   if (cut == nullptr) return d;
                                   const auto &s = cut->stats();
                                   d["seconds"] = s.seconds;
                                   d["refused"] = s.refused;
                                   d["air_cells"] = s.air_cells;
                                   d["layer_cells"] = s.layer_cells;
                                   return d;
                               })
        .def("probe_found", [](const SolverHolder &h, std::size_t p) { return h.solver->probe_found(p); },
             py::arg("probe"))
        .def("probe_in_sight", [](const SolverHolder &h, std::size_t p) { return h.solver->probe_in_sight(p); },
             py::arg("probe"))
        .def_property_readonly("source_on_face", [](const SolverHolder &h) { return h.solver->source_on_face(); })
        .def_property_readonly("probes", [](const SolverHolder &h) { return h.solver->probes(); })
        .def("run", &run, py::arg("signal"))
        .def("reset", [](SolverHolder &h) { h.solver->reset(); })
        .def("layout", &layout);

    py::class_<FitHolder, std::shared_ptr<FitHolder>>(m, "CutFit")
        .def(py::init(&make_fit), py::arg("vertices"), py::arg("faces"), py::arg("face_material"),
             py::arg("materials"), py::arg("origin"), py::arg("cell"), py::arg("nx"), py::arg("ny"), py::arg("nz"),
             py::arg("source"), py::arg("layer") = 0, py::arg("threads") = 0)
        .def("cut_cells", &fit_cells)
        .def("cut_air", [](const FitHolder &h) { return to_numpy(h.cut->air()); })
        .def("cut_widths",
             [](const FitHolder &h) {
                 return py::make_tuple(to_numpy(h.cut->widths(0)), to_numpy(h.cut->widths(1)), to_numpy(h.cut->widths(2)));
             })
        .def_property_readonly("cut_stats",
                               [](const FitHolder &h) {
                                   const auto &st = h.cut->stats();
                                   py::dict d;
                                   d["cubes"] = st.cubes;
                                   d["regions"] = st.regions;
                                   d["squares"] = st.squares;
                                   d["ties"] = st.ties;
                                   d["dropped_area"] = st.dropped_area;
                                   d["diagonal_area"] = st.diagonal_area;
                                   d["far_volume"] = st.far_volume;
                                   d["farthest"] = st.farthest;
                                   d["air_cells"] = st.air_cells;
                                   d["seconds"] = st.seconds;
                                   return d;
                               })
        .def(
            "cut_points",
            [](const FitHolder &h, const CArray<double> &source, const CArray<double> &probes, std::size_t per_listener) {
                const std::vector<as::Vec3> src = points_of(source, "source"), ps = points_of(probes, "probes");
                if (src.size() != 1) throw std::invalid_argument("one source point");
                const auto &n = h.cut->shape();
                const auto fp = as::WaveSolver::FittedStencil(*h.cut, n[0], n[1], n[2], h.cut->cell())
                                    .points(src[0], ps, per_listener);
                auto cells = [](const std::vector<std::pair<std::size_t, double>> &v) {
                    py::list l;
                    for (const auto &[i, w] : v) l.append(py::make_tuple(i, w));
                    return l;
                };
                py::dict out;
                out["source"] = cells(fp.source);
                py::list pl;
                for (const auto &p : fp.probes) pl.append(cells(p));
                out["probes"] = pl;
                return out;
            },
            py::arg("source"), py::arg("probes"), py::arg("probes_per_listener") = 1);
}
