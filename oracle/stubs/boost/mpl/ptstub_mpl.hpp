/* Minimal stand-in for the three Boost.MPL templates the reference uses as compile-time type
   maps (solver/array.h:24-26, 95-129; patchtable/patchtable.h:150-161).  Boost is not installed
   in this environment; the oracle build only needs map/pair/integral_c/at lookups. */
#ifndef PTSTUB_BOOST_MPL_HPP
#define PTSTUB_BOOST_MPL_HPP
namespace boost { namespace mpl {
template<class T, T N> struct integral_c { static const T value = N; typedef integral_c type; };
template<class K, class V> struct pair { typedef K first; typedef V second; };
template<class... Ps> struct map {};
template<class M, class K> struct at;
template<class K, class P0, class... Ps> struct at<map<P0, Ps...>, K> : at<map<Ps...>, K> {};
template<class K, class V, class... Ps> struct at<map<pair<K, V>, Ps...>, K> { typedef V type; };
}}
#endif
