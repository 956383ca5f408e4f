// Instantiation unit: REAL=double, operator id 3 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 3
#include "stage_inst.cuh"
