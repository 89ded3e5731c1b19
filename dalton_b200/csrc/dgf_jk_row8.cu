// Row 8 (bra class 8) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(8)
