/* Core API: environment, parameters, drivers, stages (reference src/include/c/isvd/core.h). */
#ifndef ISVD_CORE_H_
#define ISVD_CORE_H_

#include <isvd/core/env.h>
#include <isvd/core/param.h>
#include <isvd/core/s_driver.h>
#include <isvd/core/d_driver.h>
#include <isvd/core/s_stage.h>
#include <isvd/core/d_stage.h>

#endif  /* ISVD_CORE_H_ */
