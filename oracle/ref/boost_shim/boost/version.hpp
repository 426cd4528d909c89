// Project-written stand-in: reports a Boost version new enough for pe's feature checks.
#ifndef PE_ORACLE_SHIM_VERSION_HPP
#define PE_ORACLE_SHIM_VERSION_HPP
#define BOOST_VERSION 105800
#endif
