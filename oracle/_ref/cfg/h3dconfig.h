#define WITH_HEX
#define PACKAGE_NAME "Hermes3D"
#define PACKAGE_VERSION "0.0.1"
#define PACKAGE_STRING "Hermes3D v0.0.1"
#define PACKAGE_BUGREPORT ""
#define PACKAGE_TARNAME "hermes3d"
