// Row 5 (bra class 5) of the two-electron gradient kernel table.
#include "dgf_grad_kernel.cuh"

DGF_GRAD_ROW(5)
