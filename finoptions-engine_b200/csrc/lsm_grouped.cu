// lsm_grouped.cu - grouped / row-addressed batches (price_lsm_call_grouped_batch).
#include <cuda_runtime.h>

#include "../../include/finoptions_cuda.h"
#include "host.h"

using namespace fo;

extern "C" {

int fo_price_lsm_grouped_f64(fo_executor*, const fo_lsm_grouped_request*, fo_batch_result_columns*, fo_error* err) {
    write_error(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "grouped pricing is not available in this build"));
    return FO_ERR_EXECUTION;
}

int fo_price_lsm_batch_f64(fo_executor*, const fo_lsm_grouped_request*, fo_batch_result_columns*, fo_error* err) {
    write_error(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "row batch pricing is not available in this build"));
    return FO_ERR_EXECUTION;
}

}  // extern "C"
