// gdem_kernels.cuh -- launcher declarations of the DEM step kernels.
#pragma once
#include "gdem_device.cuh"

namespace gdem {

// gdem_integrate.cu
void launch_key(DevState const& S, double h, double dt, int pre_kick, double pre_h, cudaStream_t st);
void launch_move_gather(DevState const& S, int moving, double h, double dt, int pre_kick,
                        double pre_h, cudaStream_t st);
void launch_bin(DevState const& S, cudaStream_t st);
void launch_kick(DevState const& S, double h, cudaStream_t st);
void launch_scan(DevState const& S, cudaStream_t st);
void launch_place(DevState const& S, cudaStream_t st);
void launch_cellsort(DevState const& S, cudaStream_t st);
void launch_scatter_by_id(DevState const& S, double* x, double* v, double* w, double* wbf,
                          double* q, double* F, double* T, int id_base, cudaStream_t st);
void launch_basis_by_id(DevState const& S, double* out, int id_base, cudaStream_t st);
void launch_cells_by_id(DevState const& S, int* ijk, int id_base, cudaStream_t st);
void launch_hist_zero_cumulative(HistTable const& t, int fp64, cudaStream_t st);
void launch_load_state(DevState const& S, const double* x, const double* v, const double* w,
                       const double* wbf, const double* q, const double* F, const double* T,
                       const int* type_by_id, const int* inst_by_id, cudaStream_t st);
void launch_vstats(DevState const& S, double* part, double* out, cudaStream_t st);
void launch_pair_counts(DevState const& S, unsigned long long* out, cudaStream_t st);

// gdem_contact64.cu (FP64 mode)
void launch_pairs64(DevState const& S, cudaStream_t st);
void launch_forces64(DevState const& S, cudaStream_t st);

// gdem_contact32.cu (FP32-split mode)
void launch_pairs32(DevState const& S, cudaStream_t st);
void launch_forces32(DevState const& S, cudaStream_t st);

}  // namespace gdem
