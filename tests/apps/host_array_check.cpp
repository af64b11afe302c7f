// Host-side use of HostDeviceArray1D (myHostDeviceArray.h): pushes, inserts,
// erases, resizes, moves and sizes, printed so that builds against this
// library's header and the reference's can be compared.  No device call is
// made, so no GPU is needed.
#include <cstdio>
#include <utility>

#include "CUDAKernelFunction/myUtility/myHostDeviceArray.h"

template <class A>
static void show(const char* tag, const A& a)
{
    std::printf("%s host %zu device %zu gb %.3f:", tag, a.hostSize(), a.deviceSize(), a.deviceMemoryGB());
    for (const auto& v : a.hostRef()) std::printf(" %g", (double)v);
    std::printf(" ptr %d\n", a.d_ptr == nullptr ? 0 : 1);
}

int main()
{
    HostDeviceArray1D<double> a;
    show("empty", a);
    for (int i = 0; i < 5; ++i) a.pushHost(i * 1.5);
    show("push", a);
    a.insertHost(2, -1.0);
    a.insertHost(100, 9.0);
    show("insert", a);
    a.eraseHost(0);
    a.eraseHost(100);
    show("erase", a);
    a.resizeHost(8);
    show("resize", a);
    a.reserveHost(64);
    a.setHost({3.0, 2.0, 1.0});
    show("set", a);
    HostDeviceArray1D<double> b(std::move(a));
    show("moved-from", a);
    show("moved-to", b);
    HostDeviceArray1D<int> c;
    c.pushHost(7);
    c = HostDeviceArray1D<int>();
    show("reassigned", c);
    b.clearHost();
    show("clear", b);
    return 0;
}
