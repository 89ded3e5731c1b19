// Row 3 (bra class 3) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(3)
