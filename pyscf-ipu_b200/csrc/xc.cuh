#pragma once
#include "device_plan.cuh"
int b2_grid_setup(B2PlanDev &P, const long long *grid_off_host);
void b2_grid_free(B2PlanDev &P);
int b2_launch_ao_eval(const B2PlanDev &P, int precision, const double *coords, void *ao, cudaStream_t st);
int b2_launch_xc(const B2PlanDev &P, int precision, const int *active, const void *ao,
                 const double *w, const double *D, double *V, double *exc, cudaStream_t st);
int b2_launch_xc_direct(const B2PlanDev &P, int precision, const int *active, const double *coords,
                        const double *w, const double *D, double *V, double *exc, cudaStream_t st);
int b2_launch_xc_tc(const B2PlanDev &P, const int *active, const double *coords, const double *w,
                    const double *D, double *V, double *exc, cudaStream_t st);
// per-bucket persistent tensor-core XC (default float32 implementation)
int b2_launch_xc_tq(const B2PlanDev &P, const int *active, const double *coords, const double *w,
                    const double *D, double *V, double *exc, cudaStream_t st);
int b2_xc_tc_status_read(int reset);
int b2_zero_exc(const B2PlanDev &P, const int *active, double *exc, cudaStream_t st);
int b2_sym_v(const B2PlanDev &P, const int *active, double *V, cudaStream_t st);
int b2_xc_set_tpc(B2PlanDev &P, int tpc);
