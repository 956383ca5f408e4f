// Instantiation unit: REAL=double, operator id 0 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 0
#include "stage_inst.cuh"
