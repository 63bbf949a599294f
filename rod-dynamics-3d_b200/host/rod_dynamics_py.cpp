// rod_dynamics_py.cpp - the reference's Python module surface
// (src/python/rod_dynamics_py.cpp:93-103: Simulator(scene_path,
// init_csv_path="", quiet=True), step(steps=1), diagnostics(), rods()) over
// librodgpu.  Errors from the library become Python exceptions.
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "simulator.hpp"

namespace py = pybind11;

namespace {

std::vector<double> v3(const std::vector<double>& a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

py::dict rod_dict(const rgsim::Simulator& s, int i) {
  const auto &x = s.x(), &q = s.q(), &v = s.v(), &w = s.w(), &f = s.f(), &t = s.tau();
  py::dict d;
  d["position"] = v3(x, i);
  d["orientation_wxyz"] = std::vector<double>{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
  d["linear_velocity"] = v3(v, i);
  d["angular_velocity"] = v3(w, i);
  d["force"] = v3(f, i);
  d["torque"] = v3(t, i);
  const double m = s.mass(i);
  d["mass"] = m;
  d["inverse_mass"] = m > 0 ? 1.0 / m : 0.0;
  d["friction"] = s.config().model == RG_MODEL_NSC ? s.config().nsc_mu : s.config().soft_mu;
  d["restitution"] = s.restitution(i);
  d["shape"] = "capsule";
  d["radius"] = s.radius(i);
  d["half_height"] = s.half_height(i);
  double a[3], b[3];
  s.endpoints(i, a, b);
  d["endpoint_a"] = std::vector<double>{a[0], a[1], a[2]};
  d["endpoint_b"] = std::vector<double>{b[0], b[1], b[2]};
  return d;
}

}  // namespace

PYBIND11_MODULE(rod_dynamics_py, m) {
  m.doc() = "Rod dynamics on B200: the reference's Simulator surface over librodgpu";
  py::class_<rgsim::Simulator>(m, "Simulator")
      .def(py::init<const std::string&, const std::string&, bool>(), py::arg("scene_path"),
           py::arg("init_csv_path") = std::string(), py::arg("quiet") = true)
      .def("step", &rgsim::Simulator::step, py::arg("steps") = 1, py::call_guard<py::gil_scoped_release>())
      .def("enable_csv", &rgsim::Simulator::enable_csv, py::arg("path") = std::string("profile.csv"),
           "Profile CSV of every frame, the reference App's columns (main.cpp:3276-3355).")
      .def("enable_network", &rgsim::Simulator::enable_network, py::arg("path") = std::string("network.csv"),
           py::arg("stride") = 1, py::arg("max_frames") = 0,
           "NSC contact network CSV every stride frames (main.cpp:3620-3700).")
      .def("diagnostics",
           [](const rgsim::Simulator& s) {
             py::dict d;
             d["frame_index"] = s.frame_index();
             d["dt"] = s.dt();
             d["last_ke"] = s.last_ke();
             d["last_hit_count"] = s.last_hit_count();
             d["last_island_count"] = 0;  // contact islands are not formed on this path
             d["rod_count"] = s.rod_count();
             return d;
           })
      .def("rods",
           [](const rgsim::Simulator& s) {
             std::vector<py::dict> out;
             out.reserve(s.rod_count());
             for (int i = 0; i < s.rod_count(); ++i) out.push_back(rod_dict(s, i));
             return out;
           })
      .def("stats",
           [](const rgsim::Simulator& s) {
             const rg_step_stats& t = s.last_stats();
             py::dict d;
             d["contacts"] = t.contacts;
             d["psor_sweeps"] = t.psor_sweeps;
             d["residual"] = t.residual;
             d["max_residual"] = t.max_residual;
             d["not_converged"] = t.not_converged;
             d["kinetic_energy"] = t.kinetic_energy;
             d["potential_energy"] = t.potential_energy;
             d["device_ms"] = t.device_ms;
             return d;
           },
           "Statistics of the last step() call (this library's addition).");
}
