// Instantiation unit: REAL=double, operator id 1 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 1
#include "stage_inst.cuh"
