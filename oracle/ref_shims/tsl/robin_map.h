/* The reference's robin_map submodule is not vendored; std::unordered_map has the interface it
 * uses (operator[], find, erase, bucket_count).  Only iteration order differs. */
#ifndef SBP_REF_ROBIN_MAP_SHIM_H
#define SBP_REF_ROBIN_MAP_SHIM_H
#include <unordered_map>
namespace tsl {
template <class Key, class T>
using robin_map = std::unordered_map<Key, T>;
}
#endif
