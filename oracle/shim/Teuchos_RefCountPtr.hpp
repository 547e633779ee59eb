#ifndef SHIM_TEUCHOS_RCP
#define SHIM_TEUCHOS_RCP
#include <memory>
namespace Teuchos {
template <class T> class RefCountPtr {
public:
  RefCountPtr() {}
  explicit RefCountPtr(T* p) : p_(p) {}
  T* operator->() const { return p_.get(); }
  T& operator*() const { return *p_; }
  T* get() const { return p_.get(); }
  bool is_null() const { return !p_; }
private:
  std::shared_ptr<T> p_;
};
template <class T> RefCountPtr<T> rcp(T* p) { return RefCountPtr<T>(p); }
template <class T> using RCP = RefCountPtr<T>;
}
#endif
