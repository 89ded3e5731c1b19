// Row 2 (bra class 2) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(2)
