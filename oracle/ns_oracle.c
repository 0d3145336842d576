/* ns_oracle.c -- CPU restatement of the RK3 sub-step (filled in with the
 * stepper oracle).  TEST INFRASTRUCTURE ONLY. */
#include "oracle.h"
