// Project-written stand-in: the reference's CPU entry includes jaxlib's
// c_api.h but uses nothing from it (the XLA_FFI_* registration lives in
// pymdp/ffi/registration/xla_register.cc, which is not compiled here).
#pragma once
