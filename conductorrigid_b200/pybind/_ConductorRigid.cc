// _ConductorRigid.cc -- Python module of the C++ force compute, with the methods the
// reference exports through Boost.Python (cppmodule/module.cc:9-13,
// ConductorRigid.cc:624-633): SetParams, UpdateField, UpdateParams, OutputData, plus
// computeForces (called by HOOMD's integrator in the reference) and result accessors.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <memory>
#include <stdexcept>

#include "../../include/ConductorRigid.hpp"

namespace py = pybind11;
using conductor_rigid::ConductorRigid;
using conductor_rigid::Options;
using conductor_rigid::SystemView;

namespace {

template <typename T> py::array_t<T> exact(py::object o, const char *name) {
    auto a = py::array_t<T>::ensure(o);
    if (!a || !(a.flags() & py::array::c_style)) throw std::invalid_argument(std::string(name) + " must be a C-contiguous array");
    if (!py::isinstance<py::array_t<T>>(o)) throw std::invalid_argument(std::string(name) + " has the wrong dtype");
    return a;
}

std::array<double, 3> vec3(py::sequence s) {
    if (py::len(s) != 3) throw std::invalid_argument("field must have three components");
    return {s[0].cast<double>(), s[1].cast<double>(), s[2].cast<double>()};
}

// Keeps the system's arrays alive for the C++ object that points into them.
struct PyConductorRigid {
    py::array_t<double> pos, charge, body_pos, box;
    py::array_t<uint8_t> rigid;
    std::unique_ptr<ConductorRigid> cr;

    PyConductorRigid(py::object system, py::sequence body, py::sequence charge_list, py::sequence field, double xi,
                     double errortol, const std::string &fileprefix, int period, int t0, py::dict options) {
        pos = exact<double>(system.attr("pos"), "system.pos");
        charge = exact<double>(system.attr("charge"), "system.charge");
        body_pos = exact<double>(system.attr("body_pos"), "system.body_pos");
        rigid = exact<uint8_t>(system.attr("rigid"), "system.rigid");
        box = exact<double>(system.attr("L"), "system.L");
        SystemView v;
        v.n_beads = (int)charge.size();
        v.pos = pos.data();
        v.charge = charge.mutable_data();
        v.n_bodies = (int)rigid.size();
        v.body_pos = body_pos.data();
        v.rigid = rigid.data();
        if (box.size() != 3 || pos.size() != 3 * (py::ssize_t)v.n_beads || body_pos.size() != 3 * (py::ssize_t)v.n_bodies)
            throw std::invalid_argument("inconsistent system array sizes");
        for (int k = 0; k < 3; ++k) v.L[k] = box.data()[k];
        std::vector<uint32_t> b;
        for (auto x : body) b.push_back(x.cast<uint32_t>());
        std::vector<double> q;
        for (auto x : charge_list) q.push_back(x.cast<double>());
        Options o;
        for (auto item : options) {
            const std::string k = item.first.cast<std::string>();
            py::handle v2 = item.second;
            if (k == "grid") {
                if (py::isinstance<py::int_>(v2)) {
                    o.grid[0] = o.grid[1] = o.grid[2] = v2.cast<int>();
                } else {
                    auto g = v2.cast<std::vector<int>>();
                    if (g.size() != 3) throw std::invalid_argument("grid must be an int or three ints");
                    for (int d = 0; d < 3; ++d) o.grid[d] = g[d];
                }
            } else if (k == "support") o.support = v2.cast<int>();
            else if (k == "rcut") o.rcut = v2.cast<double>();
            else if (k == "gmres_tol") o.gmres_tol = v2.cast<double>();
            else if (k == "restart") o.restart = v2.cast<int>();
            else if (k == "maxiter") o.maxiter = v2.cast<int>();
            else if (k == "precision") o.precision = v2.cast<int>();
            else if (k == "precond") o.precond = v2.cast<int>();
            else if (k == "learned") o.learned = v2.cast<int>();
            else throw std::invalid_argument("unknown option " + k);
        }
        cr.reset(new ConductorRigid(v, b, q, vec3(field), xi, errortol, fileprefix, period, t0, o));
    }
};

}  // namespace

PYBIND11_MODULE(_ConductorRigid, m) {
    m.doc() = "C++ force compute of the B200 conductor solve (reference surface)";
    py::class_<PyConductorRigid>(m, "ConductorRigid")
        .def(py::init<py::object, py::sequence, py::sequence, py::sequence, double, double, const std::string &, int,
                      int, py::dict>(),
             py::arg("system"), py::arg("body"), py::arg("charge"), py::arg("field"), py::arg("xi"),
             py::arg("errortol"), py::arg("fileprefix"), py::arg("period"), py::arg("t0"),
             py::arg("options") = py::dict())
        .def("SetParams", [](PyConductorRigid &s) { s.cr->SetParams(); })
        .def("UpdateField", [](PyConductorRigid &s, py::sequence f) { s.cr->UpdateField(vec3(f)); })
        .def("UpdateParams", [](PyConductorRigid &s, py::sequence f, const std::string &prefix, int period,
                                int t0) { s.cr->UpdateParams(vec3(f), prefix, period, t0); })
        .def("OutputData", [](PyConductorRigid &s, unsigned int t) { s.cr->OutputData(t); })
        .def("computeForces", [](PyConductorRigid &s, unsigned int t) {
            py::gil_scoped_release release;
            s.cr->computeForces(t);
        })
        .def_property_readonly("forces", [](PyConductorRigid &s) {
            const auto &f = s.cr->forces();
            py::array_t<double> a({(py::ssize_t)(f.size() / 3), (py::ssize_t)3});
            std::copy(f.begin(), f.end(), a.mutable_data());
            return a;
        })
        .def_property_readonly("potentials", [](PyConductorRigid &s) {
            const auto &p = s.cr->potentials();
            py::array_t<double> a((py::ssize_t)p.size());
            std::copy(p.begin(), p.end(), a.mutable_data());
            return a;
        })
        .def_property_readonly("stats", [](PyConductorRigid &s) {
            const cr_solve_stats &st = s.cr->stats();
            py::dict d;
            d["iterations"] = st.iterations;
            d["restarts"] = st.restarts;
            d["refinements"] = st.refinements;
            d["matvecs_fp64"] = st.matvecs_fp64;
            d["matvecs_fp32"] = st.matvecs_fp32;
            d["converged"] = st.converged;
            d["initial_residual"] = st.initial_residual;
            d["final_residual"] = st.final_residual;
            d["solve_ms"] = st.solve_ms;
            return d;
        })
        .def_property_readonly("derived", [](PyConductorRigid &s) {
            const cr_derived d = s.cr->derived();
            py::dict o;
            o["grid"] = std::vector<int>{d.grid[0], d.grid[1], d.grid[2]};
            o["support"] = d.support;
            o["rcut"] = d.rcut;
            o["eta"] = std::vector<double>{d.eta[0], d.eta[1], d.eta[2]};
            return o;
        });
}
