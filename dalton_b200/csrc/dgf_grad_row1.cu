// Row 1 (bra class 1) of the two-electron gradient kernel table.
#include "dgf_grad_kernel.cuh"

DGF_GRAD_ROW(1)
