/* Build shim for compiling the reference's stage code on the host: the
 * reference holds its plan implementations through boost::shared_ptr
 * (e.g. Pipeline/hd/remove_baseline.h:13); std::shared_ptr has the same
 * meaning for that use. */
#pragma once
#include <memory>
namespace boost { using std::shared_ptr; }
