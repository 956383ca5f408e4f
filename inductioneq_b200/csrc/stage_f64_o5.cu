// Instantiation unit: REAL=double, operator id 5 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 5
#include "stage_inst.cuh"
