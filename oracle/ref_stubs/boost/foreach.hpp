// Minimal stand-in for boost/foreach.hpp used only to compile the reference
// solver as a CPU oracle: maps BOOST_FOREACH onto a C++11 range-for.
#ifndef ORACLE_STUB_BOOST_FOREACH_HPP
#define ORACLE_STUB_BOOST_FOREACH_HPP
#define BOOST_FOREACH(decl, range) for (decl : range)
#define BOOST_REVERSE_FOREACH(decl, range) for (decl : range)
#endif
