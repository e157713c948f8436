/* See ptree.hpp in this directory: read_json and json_parser_error come from there. */
#include "ptree.hpp"
