"""The OpenMM adapter (include/dmffb200_openmm.hpp) against a fake CUDA-platform context, on the
CPU: the device view it hands to dmffb_md_force_execute (posq and its precision, the fixed-point
force buffer, the atom-index array, atom counts, the box rows in nm, the stream) and the
includeForces / includeEnergy semantics of the reference plugin's execute
(backend/openmm_dmff_plugin/platforms/cuda/src/CudaDMFFKernels.cpp:118-220).  The library calls
are stubs that record what they receive; the GPU behaviour is tested in test_gpu_md_force.py."""
import os
import shutil
import subprocess
import tempfile

import pytest

INC = os.path.join(os.path.dirname(__file__), "..", "include")

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "dmffb200_openmm.hpp"

static dmffb_md_context g_seen;
static int g_include_forces = -1, g_created = 0, g_destroyed = 0;
struct dmffb_md_force { int dummy; };
static dmffb_md_force g_force;
extern "C" int dmffb_md_force_create(const dmffb_admp_desc* d, const double*, const double*, const double*,
                                     dmffb_md_force** out) { g_created = d->n_atoms; *out = &g_force; return 0; }
extern "C" int dmffb_md_force_execute(dmffb_md_force*, const dmffb_md_context* c, int32_t inc, double* e) {
    g_seen = *c; g_include_forces = inc; *e = -123.5; return DMFFB_NOT_CONVERGED; }
extern "C" void dmffb_md_force_destroy(dmffb_md_force*) { ++g_destroyed; }

struct Vec3 { double v[3]; double operator[](int k) const { return v[k]; } };
struct Array { unsigned long long p; unsigned long long getDevicePointer() const { return p; } };
struct FakeContext {
    Array posq{0x1000}, force{0x2000}, index{0x3000};
    bool dbl = true; int current = 0;
    Array& getPosq() { return posq; }
    Array& getForce() { return force; }
    Array& getAtomIndexArray() { return index; }
    int getNumAtoms() const { return 81; }
    int getPaddedNumAtoms() const { return 96; }
    bool getUseDoublePrecision() const { return dbl; }
    void getPeriodicBoxVectors(Vec3& a, Vec3& b, Vec3& c) const {
        a = Vec3{{3.1, 0.0, 0.0}}; b = Vec3{{0.2, 3.2, 0.0}}; c = Vec3{{-0.1, 0.3, 3.3}}; }
    void* getCurrentStream() const { return (void*)0x4000; }
    void setAsCurrent() { ++current; }
};

int main() {
    dmffb_admp_desc d = {};
    d.n_atoms = 81;
    double q[81 * 9] = {0}, pol[81] = {0}, th[81] = {0};
    {
        dmffb::OpenMMForceAdapter<FakeContext, Vec3> f(d, q, pol, th);
        FakeContext cu;
        double e1 = f.execute(cu, true, true);
        printf("e1 %.3f inc %d current %d\n", e1, g_include_forces, cu.current);
        printf("posq %llx dbl %d force %llx index %llx n %d padded %d stream %llx\n",
               (unsigned long long)(uintptr_t)g_seen.posq, g_seen.posq_double,
               (unsigned long long)(uintptr_t)g_seen.force_buffer, (unsigned long long)(uintptr_t)g_seen.atom_index,
               g_seen.num_atoms, g_seen.padded_num_atoms, (unsigned long long)(uintptr_t)g_seen.stream);
        printf("box");
        for (int k = 0; k < 9; ++k) printf(" %.2f", g_seen.box_nm[k]);
        printf("\n");
        cu.dbl = false;
        double e2 = f.execute(cu, false, false);
        printf("e2 %.3f inc %d dbl %d\n", e2, g_include_forces, g_seen.posq_double);
    }
    printf("created %d destroyed %d\n", g_created, g_destroyed);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_openmm_adapter_hands_the_platform_arrays_to_the_library():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        open(src, "w").write(PROGRAM)
        exe = os.path.join(d, "t")
        subprocess.run(["g++", "-std=c++17", "-I", INC, src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[0] == "e1 -123.500 inc 1 current 1"  # NOT_CONVERGED is a warning: the energy comes back
    assert out[1] == "posq 1000 dbl 1 force 2000 index 3000 n 81 padded 96 stream 4000"
    assert out[2] == "box 3.10 0.00 0.00 0.20 3.20 0.00 -0.10 0.30 3.30"  # rows = lattice vectors, nm
    assert out[3] == "e2 0.000 inc 0 dbl 0"  # includeEnergy false -> 0, as the plugin; float4 posq
    assert out[4] == "created 81 destroyed 1"
