// Row 3 (bra class 3) of the two-electron gradient kernel table.
#include "dgf_grad_kernel.cuh"

DGF_GRAD_ROW(3)
