// 2PL family: tpl_nw, tpl_wd, slow_tpl_nw, slow_tpl_wd.
#include "cc_launch.cuh"
GCC_FAMILY(tpl, S_TPL_NW, S_TPL_WD, S_SLOW_TPL_NW, S_SLOW_TPL_WD)
