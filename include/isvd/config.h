/* Version of the iSVD API this library implements (reference CMakeLists.txt:9-11). */
#ifndef ISVD_CONFIG_H_
#define ISVD_CONFIG_H_

#define ISVD_MAJOR_VERSION 1
#define ISVD_MINOR_VERSION 3
#define ISVD_PATCH_VERSION 2
#define ISVD_VERSION "1.3.2"

#define ISVD_B200_VERSION "0.1.0"

#endif  /* ISVD_CONFIG_H_ */
