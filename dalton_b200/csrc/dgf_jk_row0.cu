// Row 0 (bra class 0) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(0)
