// Row 7 (bra class 7) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(7)
