"""Reference constants, restated with the reference's names and values.

Sources: ppm/src/ppm_param.h (kernel ids :405-407, boundary conditions :333-338,
map types :183-192, error severities :372-375) and ppm/src/ppm_error.h
(error numbers).
"""

# kernels (ppm_param.h:405-407)
ppm_param_rmsh_kernel_bsp2 = 1
ppm_param_rmsh_kernel_mp4 = 2
ppm_param_rmsh_kernel_m3p6 = 3

# boundary conditions (ppm_param.h:333-338)
ppm_param_bcdef_periodic = 1
ppm_param_bcdef_freespace = 2
ppm_param_bcdef_symmetry = 3
ppm_param_bcdef_neumann = 4
ppm_param_bcdef_dirichlet = 5
ppm_param_bcdef_robin = 6

# mapping types (ppm_param.h:183-192)
ppm_param_map_pop = 1
ppm_param_map_push = 2
ppm_param_map_send = 4
ppm_param_map_ghost_get = 5
ppm_param_map_ghost_put = 6
ppm_param_map_init = 10

# error severities (ppm_param.h:372-375)
ppm_error_notice = -4
ppm_error_warning = -3
ppm_error_error = -2
ppm_error_fatal = -1

# error numbers (ppm_error.h)
ppm_err_alloc = 101
ppm_err_dealloc = 102
ppm_err_part_range = 402
ppm_err_part_unass = 405
ppm_err_index_corr = 410
ppm_err_wrong_dim = 501
ppm_err_argument = 503
ppm_err_sub_failed = 602
ppm_err_ppm_noinit = 903

# kernel half-support (ppm_interp_p2m.f:328 overwrite of ppm_module_data_rmsh.f:49-50)
ppm_rmsh_kernelsize = (1, 2, 2, 4)
