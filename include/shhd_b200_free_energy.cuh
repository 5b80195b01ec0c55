/* Free-energy styles compiled into the engine as device plugins.
 *
 * The counterpart, for the step's hot path, of the reference's free-energy plugin seam: a style
 * registered by name (FreeEnergyRegistry::register_free_energy_style / get_free_energy,
 * src/model_free_energy_registry.h:65-85) whose object answers the per-point virtual
 * FreeEnergy::physical_chemical_potential (src/model_free_energy.h:27-52).  Here a style is a
 * struct whose static member templates the kernels inline at the point where the row pass forms
 * its products; the engine looks a style up by name when it parses `model free_energy <name>`.
 *
 *   struct MyStyle {
 *       static constexpr const char* kName = "my_style";       // `model free_energy my_style ...`
 *       static constexpr int kParams = 2;                      // at most SHHD_MAX_FE_PARAMS
 *       // script keys of the parameters, in order: "k[]" takes one value per order parameter
 *       // (written k[0], k[1], ...), "k" one value
 *       static constexpr const char* kKeys[kParams] = {"u[]", "g"};
 *       // physical chemical potential of order parameter a at one point: psi_a its value there,
 *       // psi[0..n-1] all order parameters there; p(k, b) parameter k of order parameter b
 *       // (a one-value key: p(k, 0))
 *       template <typename T, typename Params>
 *       __device__ static T mu(int a, T psi_a, const T* psi, int n, const Params& p);
 *       // the free-energy density of that physical part at one point (the energy measure)
 *       template <typename T, typename Params>
 *       __device__ static T density(const T* psi, int n, const Params& p);
 *   };
 *
 * psi holds SHHD_MAX_ORDER_PARAMETERS values in registers: loop over it with that compile-time
 * bound (#pragma unroll, `if (b < n)`), so that no index is a run-time one.
 *
 * The linear part (a[a] + b[a] k^2) psi_a is applied in Fourier space, with the keys a[] and b[]
 * as for phi4.  A style is registered by adding it to SHHD_FREE_ENERGY_PLUGINS in the engine's
 * csrc/free_energy_plugins.h and rebuilding; styles are numbered from 1 in that list
 * (shhd_config.fe_plugin), and shhd_free_energy_plugin_count / _name list them.
 */
#ifndef SHHD_B200_FREE_ENERGY_CUH
#define SHHD_B200_FREE_ENERGY_CUH

#include "shhd_b200.h"

#endif
