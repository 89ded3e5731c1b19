// Row 5 (bra class 5) of the quartet-class kernel table.
#include "dgf_jk_inst.cuh"

DGF_JK_ROW(5)
