/* Generated by fit_erfc.py: erfc(x) ~= exp(-x^2) * sum_k c_k t^k, t = 1/(1+P x).
 * Fitted on x in [0, 3.7]; max relative error of the FP32 polynomial part 3.24e-07. */
#ifndef RGPU_ERFC_FIT_H
#define RGPU_ERFC_FIT_H
#define RGPU_ERFC_P 0.5f
#define RGPU_ERFC_XMAX 3.7f
#define RGPU_ERFC_DEG 8
#define RGPU_ERFC_MAXREL 3.239e-07
#define RGPU_ERFC_C0 -5.779241328e-04f
#define RGPU_ERFC_C1 2.913462222e-01f
#define RGPU_ERFC_C2 2.173816115e-01f
#define RGPU_ERFC_C3 5.052145720e-01f
#define RGPU_ERFC_C4 -4.662229121e-01f
#define RGPU_ERFC_C5 1.093051553e+00f
#define RGPU_ERFC_C6 -9.508326650e-01f
#define RGPU_ERFC_C7 3.654806018e-01f
#define RGPU_ERFC_C8 -5.484108627e-02f
#endif
