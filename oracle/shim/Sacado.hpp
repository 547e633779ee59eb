#ifndef SHIM_SACADO
#define SHIM_SACADO
#endif
