// Row 4 (bra class 4) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(4)
