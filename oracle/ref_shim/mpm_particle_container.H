// Stand-in for the particle container type that Source/interpolants.H names
// (reference pin only): a particle with realData/intData storage.
#ifndef EXG_REFPIN_PC_SHIM_H_
#define EXG_REFPIN_PC_SHIM_H_
#include "AMReX.H"
using namespace amrex;
struct MPMParticleContainer {
    struct ParticleType {
        double m_pos[3];
        double m_rdata[64];
        int m_idata[3];
        double &rdata(int i) { return m_rdata[i]; }
        double &pos(int d) { return m_pos[d]; }
        int &idata(int i) { return m_idata[i]; }
    };
};
#endif
