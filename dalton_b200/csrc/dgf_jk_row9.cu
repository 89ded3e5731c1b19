// Row 9 (bra class 9) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(9)
