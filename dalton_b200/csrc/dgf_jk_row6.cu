// Row 6 (bra class 6) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(6)
