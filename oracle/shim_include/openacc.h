/* Empty stand-in: with g++ the reference's OpenACC pragmas are inert and no
 * acc_* runtime call is made on the step path. */
#ifndef PFAG_SHIM_OPENACC_H
#define PFAG_SHIM_OPENACC_H
#endif
