// Instantiation unit: REAL=double, operator id 2 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 2
#include "stage_inst.cuh"
