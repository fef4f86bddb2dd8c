// ConductorRigid.cc -- the reference plugin's force-compute surface over the C ABI.
#include "../../include/ConductorRigid.hpp"

#include <algorithm>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace conductor_rigid {

ConductorRigid::ConductorRigid(const SystemView &sys, const std::vector<uint32_t> &body,
                               const std::vector<double> &charge, const std::array<double, 3> &field, double xi,
                               double errortol, const std::string &fileprefix, int period, int t0,
                               const Options &opts)
    : m_sys(sys),
      m_body(body),
      m_charge(charge),
      m_field(field),
      m_xi(xi),
      m_errortol(errortol),
      m_fileprefix(fileprefix),
      m_period(period),
      m_t0(t0),
      m_opts(opts) {
    if ((int)m_body.size() != sys.n_beads) throw std::invalid_argument("body list must have one entry per bead");
    if ((int)m_charge.size() != sys.n_bodies) throw std::invalid_argument("charge list must have one entry per body");
    if (sys.n_beads > 0 && (!sys.pos || !sys.charge)) throw std::invalid_argument("missing bead arrays");
    if (sys.n_bodies > 0 && (!sys.body_pos || !sys.rigid)) throw std::invalid_argument("missing body arrays");
    m_force.assign(3 * (size_t)sys.n_beads, 0.0);
    m_potential.assign((size_t)sys.n_bodies, 0.0);
}

ConductorRigid::~ConductorRigid() {
    if (m_h) cr_destroy(m_h);
}

void ConductorRigid::check(int status, const char *where) const {
    if (status == CR_OK) return;
    std::string msg = std::string(where) + ": " + cr_status_string(status);
    if (m_h) msg += std::string(" (") + cr_last_error(m_h) + ")";
    throw std::runtime_error(msg);
}

// Derive the method parameters for the current box, build tables, mesh and plans,
// and reset the body potentials (ConductorRigid.cc:359-366).
void ConductorRigid::SetParams() {
    cr_params p{};
    for (int k = 0; k < 3; ++k) {
        p.field[k] = m_field[k];
        p.grid[k] = m_opts.grid[k];
    }
    p.xi = m_xi;
    p.errortol = m_errortol;
    p.support = m_opts.support;
    p.rcut = m_opts.rcut;
    p.gmres_tol = m_opts.gmres_tol;
    p.restart = m_opts.restart;
    p.maxiter = m_opts.maxiter;
    p.precision = m_opts.precision;
    p.precond = m_opts.precond;
    p.learned = m_opts.learned;
    if (!m_h) {
        check(cr_create(&p, m_sys.L, &m_h), "SetParams");
        check(cr_set_topology(m_h, m_sys.n_beads, m_body.data(), m_sys.n_bodies, m_sys.rigid, m_charge.data()),
              "SetParams");
    } else {
        check(cr_set_params(m_h, &p, m_sys.L), "SetParams");
    }
    std::fill(m_potential.begin(), m_potential.end(), 0.0);
}

void ConductorRigid::UpdateField(const std::array<double, 3> &field) {
    m_field = field;
    if (m_h) check(cr_set_field(m_h, field.data()), "UpdateField");
}

void ConductorRigid::UpdateParams(const std::array<double, 3> &field, const std::string &fileprefix, int period,
                                  int t0) {
    m_field = field;
    m_fileprefix = fileprefix;
    m_period = period;
    m_t0 = t0;
}

cr_derived ConductorRigid::derived() const {
    cr_derived d{};
    if (m_h) cr_get_derived(m_h, &d);
    return d;
}

void ConductorRigid::computeForces(unsigned int timestep) {
    if (!m_h) SetParams();
    const int st = cr_compute_host(m_h, m_sys.pos, m_sys.body_pos, m_sys.charge, m_potential.data(), m_force.data(),
                                   &m_stats);
    if (st != CR_OK && st != CR_NOT_CONVERGED) check(st, "computeForces");
    if (m_period > 0 && ((int)timestep - m_t0) % m_period == 0) OutputData(timestep);  // cc:550-552
}

// ConductorRigid.cc:560-622: positions, charges and forces in tag order (bead index
// order here), ten significant digits, in <fileprefix>.<timestep, 10 digits>.txt.
void ConductorRigid::OutputData(unsigned int timestep) {
    std::ostringstream ts;
    ts << std::setw(10) << std::setfill('0') << timestep;
    const std::string filename = m_fileprefix + "." + ts.str() + ".txt";
    std::ofstream file(filename.c_str(), std::ios_base::out);
    if (!file.good()) throw std::runtime_error("Error in ConductorRigid: unable to open output file.");
    const int N = m_sys.n_beads;
    file << "Bead Position" << std::endl;
    for (int i = 0; i < N; ++i)
        file << std::setprecision(10) << m_sys.pos[3 * i] << "  " << m_sys.pos[3 * i + 1] << "  "
             << m_sys.pos[3 * i + 2] << "  " << std::endl;
    file << "Bead Charge" << std::endl;
    for (int i = 0; i < N; ++i) file << std::setprecision(10) << m_sys.charge[i] << std::endl;
    file << "Bead Force" << std::endl;
    for (int i = 0; i < N; ++i)
        file << std::setprecision(10) << m_force[3 * i] << "  " << m_force[3 * i + 1] << "  " << m_force[3 * i + 2]
             << "  " << std::endl;
}

}  // namespace conductor_rigid
