/* Test infrastructure only: empty stand-in for the CUDA samples'
 * helper_functions.h that ObitCUDASkyModel.cu includes (it uses none of it). */
#pragma once
