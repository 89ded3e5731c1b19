// Row 1 (bra class 1) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(1)
