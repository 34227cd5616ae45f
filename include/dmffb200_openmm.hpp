/*
 * dmffb200_openmm.hpp — C++ adapter between an OpenMM CUDA-platform force kernel and the
 * MD-platform force of libdmffb200 (dmffb_md_force_*, declared in dmffb200.h).
 *
 * It takes the place of the reference plugin's CudaCalcDMFFForceKernel
 * (backend/openmm_dmff_plugin/platforms/cuda/src/CudaDMFFKernels.cpp:47-220): initialize()
 * creates the engine from the system description, execute() hands the platform's device arrays
 * to the library and returns the energy.  Nothing crosses to the host per step but the box and
 * the energy.  The adapter is a template over the platform context, so it compiles without
 * OpenMM's headers; with OpenMM it is instantiated as
 *     dmffb::OpenMMForceAdapter<OpenMM::CudaContext, OpenMM::Vec3>
 * and the context type provides the members an OpenMM CudaContext has: getPosq(), getForce(),
 * getAtomIndexArray() (each with getDevicePointer()), getNumAtoms(), getPaddedNumAtoms(),
 * getUseDoublePrecision(), getPeriodicBoxVectors(Vec3&, Vec3&, Vec3&), getCurrentStream() and
 * setAsCurrent().  Positions and box arrive in nm; the force buffer receives kJ/mol/nm in the
 * platform's 2^32 fixed point; the energy is kJ/mol.
 */
#ifndef DMFFB200_OPENMM_HPP
#define DMFFB200_OPENMM_HPP

#include <cstdint>
#include <stdexcept>
#include <string>

#include "dmffb200.h"

namespace dmffb {

template <class Context, class Vec3>
class OpenMMForceAdapter {
  public:
    /* desc and parameters as dmffb_md_force_create (Angstrom, e, kJ/mol; Q_local [n*9]). */
    OpenMMForceAdapter(const dmffb_admp_desc& desc, const double* Q_local, const double* pol, const double* thole) {
        const int st = dmffb_md_force_create(&desc, Q_local, pol, thole, &force_);
        if (st != DMFFB_OK) throw std::runtime_error("dmffb_md_force_create failed with status " + std::to_string(st));
    }
    ~OpenMMForceAdapter() { dmffb_md_force_destroy(force_); }
    OpenMMForceAdapter(const OpenMMForceAdapter&) = delete;
    OpenMMForceAdapter& operator=(const OpenMMForceAdapter&) = delete;

    /* The device view of one step: posq, force buffer, atom order, box (nm) and stream. */
    static dmffb_md_context make_context(Context& cu) {
        dmffb_md_context c;
        c.posq = reinterpret_cast<const void*>(static_cast<uintptr_t>(cu.getPosq().getDevicePointer()));
        c.posq_double = cu.getUseDoublePrecision() ? 1 : 0;
        c.force_buffer = reinterpret_cast<long long*>(static_cast<uintptr_t>(cu.getForce().getDevicePointer()));
        c.atom_index = reinterpret_cast<const int32_t*>(static_cast<uintptr_t>(cu.getAtomIndexArray().getDevicePointer()));
        c.num_atoms = cu.getNumAtoms();
        c.padded_num_atoms = cu.getPaddedNumAtoms();
        Vec3 a, b, d;
        cu.getPeriodicBoxVectors(a, b, d);
        const Vec3* rows[3] = {&a, &b, &d};
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) c.box_nm[3 * r + k] = (*rows[r])[k];
        c.stream = reinterpret_cast<void*>(cu.getCurrentStream());
        return c;
    }

    /* One step, as CudaCalcDMFFForceKernel::execute: the forces are added to the platform's buffer
     * when includeForces; the energy is returned when includeEnergy (0 otherwise). */
    double execute(Context& cu, bool includeForces, bool includeEnergy) {
        cu.setAsCurrent();
        const dmffb_md_context c = make_context(cu);
        double e = 0.0;
        const int st = dmffb_md_force_execute(force_, &c, includeForces ? 1 : 0, &e);
        if (st != DMFFB_OK && st != DMFFB_NOT_CONVERGED)
            throw std::runtime_error("dmffb_md_force_execute failed with status " + std::to_string(st));
        return includeEnergy ? e : 0.0;
    }

    dmffb_md_force* handle() const { return force_; }

  private:
    dmffb_md_force* force_ = nullptr;
};

}  // namespace dmffb

#endif
