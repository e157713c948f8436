/* boost::property_tree names mapped onto the project's own ptree (deco_b200/host/ptree.hpp)
 * so that the reference's headers compile into the oracle library.  Test infrastructure only. */
#ifndef ORACLE_SHIM_BOOST_PTREE_HPP
#define ORACLE_SHIM_BOOST_PTREE_HPP
#include "deco_b200/host/ptree.hpp"
namespace boost {
namespace property_tree {
using ptree = ::deco::ptree;
using ptree_error = ::deco::ptree_error;
using json_parser_error = ::deco::json_parser_error;
using ::deco::read_json;
}  // namespace property_tree
}  // namespace boost
#endif
