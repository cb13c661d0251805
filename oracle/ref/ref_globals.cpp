/* Fortran module variables the reference drop-in reads by their Intel-mangled names
 * (src/physics/bxcompute_uwshcu_inv.cpp:18-47), defined here and set from the same constants the
 * oracle uses; plus the simulated thread indices of the HIP shim (TEST INFRASTRUCTURE ONLY). */
#include <string.h>
#include "hip/hip_runtime.h"

dim3 threadIdx, blockIdx, blockDim, gridDim;

double uwshcu_mp_xlv_, uwshcu_mp_xlf_, uwshcu_mp_xls_, uwshcu_mp_cp_, uwshcu_mp_zvir_, uwshcu_mp_r_,
    uwshcu_mp_g_, uwshcu_mp_ep2_, uwshcu_mp_p00_, uwshcu_mp_rovcp_, uwshcu_mp_rpen_;
char constituents_mp_cnst_type_[25][3];
double wv_saturation_mp_estbl_[250];
double wv_saturation_mp_tmin_, wv_saturation_mp_tmax_, wv_saturation_mp_ttrice_, wv_saturation_mp_pcf_[6],
    wv_saturation_mp_epsqs_, wv_saturation_mp_rgasv_, wv_saturation_mp_hlatf_, wv_saturation_mp_hlatv_,
    wv_saturation_mp_cp_, wv_saturation_mp_tmelt_;
bool wv_saturation_mp_icephs_;
double constituents_mp_qmin_[25];
int modal_aero_data_mp_numptr_amode_[3];

/* c22: xlv xlf xls cp zvir r g ep2 p00 rovcp rpen tmin tmax ttrice epsqs rgasv tmelt pcf1..pcf5 */
extern "C" void uwref_init(const double *c22, const double *estbl, const double *qmin25, const int *wet25)
{
    uwshcu_mp_xlv_ = c22[0]; uwshcu_mp_xlf_ = c22[1]; uwshcu_mp_xls_ = c22[2]; uwshcu_mp_cp_ = c22[3];
    uwshcu_mp_zvir_ = c22[4]; uwshcu_mp_r_ = c22[5]; uwshcu_mp_g_ = c22[6]; uwshcu_mp_ep2_ = c22[7];
    uwshcu_mp_p00_ = c22[8]; uwshcu_mp_rovcp_ = c22[9]; uwshcu_mp_rpen_ = c22[10];
    wv_saturation_mp_tmin_ = c22[11]; wv_saturation_mp_tmax_ = c22[12]; wv_saturation_mp_ttrice_ = c22[13];
    wv_saturation_mp_epsqs_ = c22[14]; wv_saturation_mp_rgasv_ = c22[15]; wv_saturation_mp_tmelt_ = c22[16];
    for (int i = 0; i < 5; i++) wv_saturation_mp_pcf_[i] = c22[17 + i];
    wv_saturation_mp_pcf_[5] = 0.0;
    wv_saturation_mp_hlatv_ = c22[0];
    wv_saturation_mp_hlatf_ = c22[1];
    wv_saturation_mp_cp_ = c22[3];
    wv_saturation_mp_icephs_ = true;
    memcpy(wv_saturation_mp_estbl_, estbl, sizeof(wv_saturation_mp_estbl_));
    for (int m = 0; m < 25; m++) {
        constituents_mp_qmin_[m] = qmin25[m];
        memcpy(constituents_mp_cnst_type_[m], wet25[m] ? "wet" : "dry", 3);
    }
    for (int j = 0; j < 3; j++) modal_aero_data_mp_numptr_amode_[j] = -100;
}
