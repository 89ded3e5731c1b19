// Row 2 (bra class 2) of the two-electron gradient kernel table.
#include "dgf_grad_kernel.cuh"

DGF_GRAD_ROW(2)
