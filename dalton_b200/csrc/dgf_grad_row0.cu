// Row 0 (bra class 0) of the two-electron gradient kernel table.
#include "dgf_grad_kernel.cuh"

DGF_GRAD_ROW(0)
