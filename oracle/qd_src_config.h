/* Minimal "config.h" for compiling QD's src/*.cpp without its configure
 * script (oracle build only). */
#define HAVE_STDLIB_H 1
#define HAVE_STRING_H 1
#define HAVE_STDINT_H 1
#define MAJOR_VERSION 2
#define MINOR_VERSION 3
#define PATCH_VERSION 23
#define PACKAGE_STRING "qd 2.3.23"
