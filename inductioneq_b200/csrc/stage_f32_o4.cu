// Instantiation unit: REAL=float, operator id 4 (see ieq_common.cuh).
#define IEQ_R float
#define IEQ_OP 4
#include "stage_inst.cuh"
