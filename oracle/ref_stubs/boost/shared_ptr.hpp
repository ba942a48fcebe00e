// Minimal stand-in for boost/shared_ptr.hpp used only to compile the
// reference solver as a CPU oracle: re-exports the std smart pointers.
#ifndef ORACLE_STUB_BOOST_SHARED_PTR_HPP
#define ORACLE_STUB_BOOST_SHARED_PTR_HPP
#include <memory>
namespace boost {
using std::shared_ptr;
using std::dynamic_pointer_cast;
using std::static_pointer_cast;
using std::const_pointer_cast;
using std::enable_shared_from_this;
}
#endif
