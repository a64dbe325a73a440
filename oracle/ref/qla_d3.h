/* qla_d3.h -- the shim's QLA types and site macros (qla.h) */
#include "qla.h"
