// coef_cast.h -- float64 population coefficients cast to the compute type.
#pragma once
#include "device_types.h"

namespace bspk {

template <typename Real>
PopCoef<Real> cast_coef(const PopCoef<double> &d) {
    PopCoef<Real> c;
#define C_(f) c.f = static_cast<Real>(d.f);
    C_(E_L) C_(I_e) C_(lower) C_(theta) C_(vreset) C_(P11ex) C_(P21ex) C_(P22ex) C_(P11in)
    C_(P21in) C_(P22in) C_(expm1_tm) C_(P30) C_(P31ex) C_(P32ex) C_(P31in) C_(P32in) C_(epsc)
    C_(ipsc) C_(eP11ex) C_(eP11in) C_(eP22) C_(eP21ex) C_(eP21in) C_(eP20) C_(one_m_eP11ex)
    C_(V_peak) C_(V_reset) C_(g_L) C_(C_m) C_(E_ex) C_(E_in) C_(Delta_T) C_(tau_w) C_(a) C_(b)
    C_(V_th) C_(tau_syn_ex) C_(tau_syn_in) C_(atol) C_(pscon_ex) C_(pscon_in) C_(v_peak_detect)
    C_(inv_C_m) C_(inv_tau_syn_ex) C_(inv_tau_syn_in) C_(inv_tau_w)
#undef C_
    for (int k = 0; k < 4; ++k) {
        c.msP11[k] = static_cast<Real>(d.msP11[k]);
        c.msP21[k] = static_cast<Real>(d.msP21[k]);
    }
    c.inv_Delta_T = d.inv_Delta_T;
    c.inv_Delta_T_hi = static_cast<float>(d.inv_Delta_T);
    c.inv_Delta_T_lo = static_cast<float>(d.inv_Delta_T - static_cast<double>(c.inv_Delta_T_hi));
    c.inv_atol = d.inv_atol;
    c.nrec = d.nrec;
    c.ref_count = d.ref_count;
    c.off = d.off;
    c.n = d.n;
    return c;
}

}  // namespace bspk
