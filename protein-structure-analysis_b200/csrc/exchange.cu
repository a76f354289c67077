// Replica exchange (parallel tempering) between temperature neighbours.
//
// The reference runs its tempering ladder as Python threads, one landscape
// segment per replica, and swaps states on the host (gui_main.py:1960-2013,
// run_landscape_segment physics_engine.cpp:2925-2951).  Here every replica
// is a system of one batch and the swap is a kernel: temperatures (and the
// step sizes adapted for them) move between systems instead of coordinates.
// Round r pairs temperature slots (t, t+1) with t ≡ r (mod 2); a pair swaps
// with probability min(1, exp((1/T_a - 1/T_b)(E_a - E_b))), E from fresh
// energy terms.  Pairs are disjoint, so one thread per pair.
#include "alma_common.cuh"

namespace alma {

__global__ void exchange_kernel(int nsys, const double *__restrict__ terms, AlmaChainState *__restrict__ mc,
                                AlmaMalaState *__restrict__ mala, int32_t *__restrict__ sys_of_temp, uint64_t seed,
                                int64_t round, unsigned long long *__restrict__ attempts,
                                unsigned long long *__restrict__ accepts) {
    const int t = 2 * (int)threadIdx.x + (int)(round & 1);
    if (t + 1 >= nsys) return;
    const int sa = sys_of_temp[t], sb = sys_of_temp[t + 1];
    const double Ta = mc[sa].temperature, Tb = mc[sb].temperature;
    const double Ea = terms[5 * (size_t)sa + 4], Eb = terms[5 * (size_t)sb + 4];
    const double log_acc = (1.0 / Ta - 1.0 / Tb) * (Ea - Eb);
    const uint32_t k0 = (uint32_t)seed ^ 0xA511E9B3u, k1 = (uint32_t)(seed >> 32);
    const Philox4 r = philox4x32_10((uint32_t)round, (uint32_t)((uint64_t)round >> 32), (uint32_t)t, 0x52455800u, k0, k1);
    const double u = u01_from(r.v[0], r.v[1]);
    const bool acc = isfinite(log_acc) && (log_acc >= 0.0 || log(u) < log_acc);
    attempts[t]++;
    if (!acc) return;
    accepts[t]++;
    // the temperature slot carries its adapted step and adaptation window
    AlmaChainState A = mc[sa], B = mc[sb];
    mc[sa].temperature = B.temperature;
    mc[sb].temperature = A.temperature;
    mc[sa].cur_max = B.cur_max;
    mc[sb].cur_max = A.cur_max;
    mc[sa].acc_win = B.acc_win;
    mc[sb].acc_win = A.acc_win;
    mc[sa].tot_win = B.tot_win;
    mc[sb].tot_win = A.tot_win;
    if (mala) {
        const double ba = mala[sa].beta, sca = mala[sa].scale;
        mala[sa].beta = mala[sb].beta;
        mala[sa].scale = mala[sb].scale;
        mala[sb].beta = ba;
        mala[sb].scale = sca;
    }
    sys_of_temp[t] = sb;
    sys_of_temp[t + 1] = sa;
}

}  // namespace alma

using namespace alma;

extern "C" int alma_replica_exchange(int32_t nsys, const double *terms, AlmaChainState *mc_states,
                                     AlmaMalaState *mala_states, int32_t *sys_of_temp, uint64_t seed, int64_t round,
                                     unsigned long long *attempts, unsigned long long *accepts, void *stream) {
    if (nsys <= 0 || !terms || !mc_states || !sys_of_temp || !attempts || !accepts || round < 0)
        return alma_set_error(ALMA_EINVAL, "alma_replica_exchange: bad arguments");
    if (nsys > 2048) return alma_set_error(ALMA_EINVAL, "alma_replica_exchange: at most 2048 replicas");
    if (nsys < 2) return ALMA_OK;
    const int pairs = nsys / 2;
    exchange_kernel<<<1, pairs, 0, (cudaStream_t)stream>>>(nsys, terms, mc_states, mala_states, sys_of_temp, seed,
                                                           round, attempts, accepts);
    ALMA_LAUNCH_CHECK("alma_replica_exchange");
    return ALMA_OK;
}
