/*
 * ref_shim.cpp -- extern "C" entry points over the reference's own sources.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile.ref together with the
 * reference files it names, straight from the reference tree, into
 * oracle/_ref/libvsref.so.  Nothing here restates reference logic: each
 * function constructs the reference class and calls its method, so tests can
 * pin the oracle's restatement against the reference's compiled code.
 *   TwoMassModel.cpp        setTwoMassModelParams / runTwoMassModel
 *   GlottalExcitations.cu   setExcitationVelocity
 *   SolverParams.cu         setBeta / setSigmaPrimeDt / setTimeStep / setSourceDirection
 *   SimulationParams.cu     SimulationParams(int srate_mul)
 */
#include "TwoMassModel.h"
#include "GlottalExcitations.h"
#include "SolverParams.h"
#include "SimulationParams.h"

#include <cstring>

extern "C" {

/* ug[i] after runTwoMassModel with supraglottal pressure p1[i]. */
int vsref_tmm(int srate_mul, const float* p1, long long n, float* ug) {
    TwoMassModel m;
    m.setTwoMassModelParams();
    for (long long i = 0; i < n; i++) {
        m.setSupraGlottalPressure(p1[i]);
        m.runTwoMassModel(srate_mul);
        ug[i] = m.getVolumeVelocity();
    }
    return 0;
}

/* GlottalExcitations::setExcitationVelocity(source_type, num_steps, dt). */
int vsref_excitation(int source_type, int num_steps, double dt, float* out) {
    GlottalExcitations g;
    g.setExcitationVelocity(source_type, num_steps, dt);
    thrust::host_vector<float> v = g.getExcitationVelocity();
    for (int i = 0; i < num_steps; i++) out[i] = v[i];
    return 0;
}

/* SolverParams tables for the given PML layer count, sigma scale and dt. */
int vsref_solver_tables(int num_pml_layers, float max_sigma_dt, float dt, float* beta13,
                        float* sigma13, float* dir4) {
    SolverParams s;
    s.setBeta(num_pml_layers);
    s.setSigmaPrimeDt(max_sigma_dt, dt, num_pml_layers);
    s.setSourceDirection();
    std::memcpy(beta13, s.getBeta(), 13 * sizeof(float));
    std::memcpy(sigma13, s.getSigmaPrimeDt(), 13 * sizeof(float));
    std::memcpy(dir4, s.getSourceDirection(), 4 * sizeof(float));
    return 0;
}

/* SolverParams::setTimeStep: number of steps for audio_dur. */
long long vsref_step_count(float audio_dur, float dt) {
    SolverParams s;
    s.setTimeStep(audio_dur, dt);
    return (long long)s.getTimeStep().size();
}

/* SimulationParams(srate_mul): {c, rho, kappa, dt, ds, max_sigma_dt,
 * pml_layers, cpl, Mw, Bw, Kw, srate}. */
int vsref_sim_params(int srate_mul, float* out12) {
    SimulationParams p(srate_mul);
    out12[0] = p.sound_speed; out12[1] = p.rho; out12[2] = p.kappa; out12[3] = p.dt;
    out12[4] = p.ds; out12[5] = p.max_sigma_dt; out12[6] = (float)p.pml_layers;
    out12[7] = p.wall_pressure_coupling_coeff; out12[8] = p.Mw; out12[9] = p.Bw;
    out12[10] = p.Kw; out12[11] = (float)p.srate;
    return 0;
}

}  // extern "C"
