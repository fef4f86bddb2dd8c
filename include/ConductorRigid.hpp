// ConductorRigid.hpp -- C++ force compute with the surface of the reference plugin's
// ConductorRigid class (cppmodule/ConductorRigid.h:21-112), on top of the C ABI in
// conductor_rigid.h.
//
// The reference derives from HOOMD's ForceCompute and reads positions, tags and rigid
// bodies from a SystemDefinition.  HOOMD is not part of this library, so the class
// reads them from a SystemView: host arrays owned by the caller, which must stay valid
// for the life of the object.  Bead charges are the warm start of every solve and are
// overwritten with the solution, as the reference overwrites HOOMD's charges
// (ConductorRigid.cu:1126-1139).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "conductor_rigid.h"

namespace conductor_rigid {

struct SystemView {
    int n_beads = 0;
    const double *pos = nullptr;        // [n_beads][3], inside the box [-L/2, L/2)
    double *charge = nullptr;           // [n_beads] warm start in, solution out
    int n_bodies = 0;
    const double *body_pos = nullptr;   // [n_bodies][3] rigid-body centres
    const uint8_t *rigid = nullptr;     // [n_bodies] 1 rigid body, 0 free bead
    double L[3] = {0, 0, 0};            // orthorhombic box edges
};

// Options the reference hard-codes or derives from errortol.
struct Options {
    int grid[3] = {0, 0, 0};  // 0: derive
    int support = 0;          // 0: derive
    double rcut = 0.0;        // 0: sqrt(-ln errortol)/xi
    double gmres_tol = 0.0;   // 0: errortol
    int restart = 0;          // 0: 10
    int maxiter = 0;          // 0: 100
    int precision = CR_FP64;
    int precond = CR_PRECOND_DIAGONAL;
    int learned = 0;
};

class ConductorRigid {
  public:
    // ConductorRigid.h:25-35: body = isolated-body tag of every bead (by tag), charge =
    // known charge of every isolated body, field = external field.
    ConductorRigid(const SystemView &sys, const std::vector<uint32_t> &body, const std::vector<double> &charge,
                   const std::array<double, 3> &field, double xi, double errortol, const std::string &fileprefix,
                   int period, int t0, const Options &opts = Options());
    ~ConductorRigid();
    ConductorRigid(const ConductorRigid &) = delete;
    ConductorRigid &operator=(const ConductorRigid &) = delete;

    void SetParams();                                              // ConductorRigid.cc:116-379
    void UpdateField(const std::array<double, 3> &field);         // ConductorRigid.cc:382-387
    void UpdateParams(const std::array<double, 3> &field, const std::string &fileprefix, int period,
                      int t0);                                     // ConductorRigid.cc:390-400
    void OutputData(unsigned int timestep);                        // ConductorRigid.cc:560-622
    void computeForces(unsigned int timestep);                     // ConductorRigid.cc:403-557

    const std::vector<double> &forces() const { return m_force; }            // [n_beads][3]
    const std::vector<double> &potentials() const { return m_potential; }    // [n_bodies]
    const cr_solve_stats &stats() const { return m_stats; }
    cr_derived derived() const;

  private:
    void check(int status, const char *where) const;
    SystemView m_sys;
    std::vector<uint32_t> m_body;
    std::vector<double> m_charge;
    std::array<double, 3> m_field;
    double m_xi, m_errortol;
    std::string m_fileprefix;
    int m_period, m_t0;
    Options m_opts;
    cr_handle *m_h = nullptr;
    std::vector<double> m_force, m_potential;
    cr_solve_stats m_stats{};
};

}  // namespace conductor_rigid
