#pragma once
#include "device_plan.cuh"
int b2_launch_fock_diis(const B2PlanDev &P, const int *active, const int *iter, double hyb,
                        int use_diis, const double *Hcore, const double *S, const double *D,
                        const double *J, const double *K, const double *Vxc, double *H,
                        double *diffJK, double *ring_err, double *ring_h, double *Bmat,
                        double *diis_err, cudaStream_t st);
int b2_launch_eigh_density(const B2PlanDev &P, const int *active, const int *iter, const double *H,
                           const double *Linv, double *D, double *mo_energy, double *C, double *ws,
                           int *sweeps, cudaStream_t st);
int b2_launch_energy(const B2PlanDev &P, const int *active, const double *D, const double *Hcore,
                     const double *diffJK, const double *exc, const double *enuc, double *out,
                     cudaStream_t st);
int b2_launch_chol_inv(const B2PlanDev &P, const double *S, double *Linv, int *status, cudaStream_t st);
int b2_launch_energy_jk(const B2PlanDev &P, const int *active, const double *D, const double *Hcore,
                        const double *J, const double *K, double hyb, const double *exc,
                        const double *enuc, double *diffJK, double *out, int *iter, cudaStream_t st);
