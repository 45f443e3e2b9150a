// Minimal stand-in for Charm++'s PUP serializer (unused by the oracle).
#ifndef OA_REF_STUB_PUP_H
#define OA_REF_STUB_PUP_H
namespace PUP {
class er {
 public:
  bool isUnpacking() const { return false; }
  template <typename T> er& operator|(T&) { return *this; }
  template <typename T> void operator()(T*, int) {}
  template <typename T> void operator()(T&) {}
};
}  // namespace PUP
#define PUParray(p, a, n) ((void)0)
#endif
