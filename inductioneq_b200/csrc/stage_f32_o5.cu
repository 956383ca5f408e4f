// Instantiation unit: REAL=float, operator id 5 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 5
#include "stage_inst.cuh"
