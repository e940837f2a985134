#pragma once
#include "device_plan.cuh"
int b2_launch_int1e(const B2PlanDev &P, double *S, double *T, double *V, cudaStream_t st);
int b2_launch_grid_build(B2PlanDev &P, int nz, const double *tmpl_host, const long long *tmpl_off_host,
                         double *coords, double *weights, cudaStream_t st);
int b2_launch_guess(const B2PlanDev &P, double *D, cudaStream_t st);
int b2_launch_enuc(const B2PlanDev &P, double *enuc, cudaStream_t st);
int b2_launch_eri_threshold(const B2PlanDev &P, int precision, void *eri, double thr, cudaStream_t st);
