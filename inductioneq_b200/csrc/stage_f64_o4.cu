// Instantiation unit: REAL=double, operator id 4 (see ieq_common.cuh).
#define IEQ_R double
#define IEQ_OP 4
#include "stage_inst.cuh"
