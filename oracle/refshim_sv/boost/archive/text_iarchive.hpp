/* Test infrastructure (reference harness only): stand-in for the Boost
 * serialization header that Matthew_Sim_CBM/includes/statevariable.hpp
 * includes.  The harness never serialises a StateVariable; the class only
 * needs boost::serialization::access declared for its friend declaration. */
#ifndef CBM_REFSHIM_BOOST_ARCHIVE_TEXT_IARCHIVE_HPP
#define CBM_REFSHIM_BOOST_ARCHIVE_TEXT_IARCHIVE_HPP
namespace boost { namespace serialization { class access; } }
#endif
