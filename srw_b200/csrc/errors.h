// Error numbers.  Those of the reference keep their values (cpp/src/core/srercode.h:20-222,
// FIRST_ERR_SRWDLL = 23000); numbers from 23900 are specific to this library.
#pragma once

#define SRWG_FIRST_ERR 23000
#define MEMORY_ALLOCATION_FAILURE (8 + SRWG_FIRST_ERR)
#define UNKNOWN_OPTICAL_ELEMENT (39 + SRWG_FIRST_ERR)
#define ERROR_IN_FFT (40 + SRWG_FIRST_ERR)
#define CAN_NOT_PROPAGATE_1D_RAD (59 + SRWG_FIRST_ERR)
#define PHOT_EN_SHOULD_BE_POSITIVE (109 + SRWG_FIRST_ERR)
#define SRWL_INCORRECT_PARAM_FOR_GAUS_BEAM_COMP (165 + SRWG_FIRST_ERR)
#define SRWL_INCORRECT_PARAM_FOR_INT_EXTR (166 + SRWG_FIRST_ERR)
#define SRWL_WFR_EXT_MODIF_FAILED (168 + SRWG_FIRST_ERR)
#define SRWL_INCORRECT_PARAM_FOR_WFR_PROP (171 + SRWG_FIRST_ERR)
#define SRWL_WFR_EXT_FUNC_NOT_DEFINED (172 + SRWG_FIRST_ERR)
#define SRWL_EXT_ARRAY_ALLOC_FAILED (188 + SRWG_FIRST_ERR)

#define SRWG_ERR_UNSUPPORTED (900 + SRWG_FIRST_ERR)     // feature outside the GPU path
#define SRWG_ERR_CUDA (901 + SRWG_FIRST_ERR)            // CUDA runtime error (text has details)
#define SRWG_ERR_NO_DEVICE (902 + SRWG_FIRST_ERR)       // no usable CUDA device
#define SRWG_ERR_BAD_ARG (903 + SRWG_FIRST_ERR)         // invalid argument to an extension entry point
#define SRWG_ERR_STATIC_LIMIT (904 + SRWG_FIRST_ERR)    // above the static scratch of srwgPropagElecFieldStatic
