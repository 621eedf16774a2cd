// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Zero-filling array allocation for the reference build. gas_layer.cc:12
// allocates tau with `new double[ml]`, and gas_layer_solve.cc:248 writes only
// tau[0..m-1]; apply_tau_bc (gas_layer.cc:28-29) and the viscous boundary
// conditions (fluid_2d.cc:295, fluid_2d_sio.cc:313) still read tau[m] and
// tau[m+1]. Zero-filling makes those reads deterministic (they read 0), which
// is the behaviour the CUDA path reproduces.
#include <cstdlib>
#include <new>

void* operator new[](std::size_t n) {
    void* p=std::calloc(n?n:1,1);
    if(p==NULL) throw std::bad_alloc();
    return p;
}
void operator delete[](void* p) noexcept {std::free(p);}
void operator delete[](void* p,std::size_t) noexcept {std::free(p);}
