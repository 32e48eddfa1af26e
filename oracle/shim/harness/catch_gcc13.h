/* Test infrastructure, force-included when compiling the reference's Catch
 * test programs unchanged.  Their array helpers declare
 *     friend void std::swap(AlignedArray<T, Align> &, AlignedArray<T, Align> &);
 *     friend void std::swap(DeviceArray<T> &, DeviceArray<T> &);
 * (scalar/test/utils.hpp:63, scalar/test/cuda_utils.hpp:24).  With GCC 13's
 * libstdc++, matching that declaration also tries the generic std::swap,
 * whose constraint asks whether the still-incomplete class is
 * move-constructible, a hard error.  Marking the two classes tuple-like makes
 * that constraint fail early (it tests "not tuple-like" first), so only the
 * helpers' own std::swap overloads remain, as with the compilers the
 * reference was written for.  Nothing else in those programs depends on
 * tuple-likeness. */
#include <type_traits>
template <typename T, unsigned Align> class AlignedArray;
template <typename T> class DeviceArray;
namespace std {
template <typename T, unsigned A> struct __is_tuple_like_impl<AlignedArray<T, A>> : true_type {};
template <typename T> struct __is_tuple_like_impl<DeviceArray<T>> : true_type {};
}  // namespace std
