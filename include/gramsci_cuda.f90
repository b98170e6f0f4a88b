! gramsci_cuda.f90 -- Fortran 2003 interface (iso_c_binding) to
! libgramsci_cuda.so, for a Fortran host such as the reference program
! (csabiu/Gramsci src/gramsci.F90).  The declarations mirror
! include/gramsci_cuda.h; see that header for the meaning of each argument.
! Arrays are passed in the reference's own layouts: points(3,N) is x,y,z
! interleaved, N2/N3/discN/discR in Fortran order with the used extents.
! Not compiled in this repository (no Fortran compiler was available).
module gramsci_cuda
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: GR_OK = 0, GR_E_ARG = -1, GR_E_CAPACITY = -2, &
                               GR_E_CUDA = -3, GR_E_TIMEOUT = -4, GR_E_UNSUPPORTED = -5
  interface
    integer(c_int) function gr_create(ctx, device) bind(c, name="gr_create")
      import :: c_ptr, c_int
      type(c_ptr) :: ctx
      integer(c_int), value :: device
    end function
    integer(c_int) function gr_destroy(ctx) bind(c, name="gr_destroy")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function gr_last_error(ctx) bind(c, name="gr_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function gr_set_catalog(ctx, xyz, w, buffer, n_data, n_rand) &
        bind(c, name="gr_set_catalog")
      import :: c_ptr, c_int, c_int64_t, c_double, c_int32_t
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: xyz(*), w(*)
      integer(c_int32_t), intent(in) :: buffer(*)
      integer(c_int64_t), value :: n_data, n_rand
    end function
    integer(c_int) function gr_set_bins(ctx, rmin, rmax, nbins, nmu, logbins) &
        bind(c, name="gr_set_bins")
      import :: c_ptr, c_int, c_double, c_int32_t
      type(c_ptr), value :: ctx
      real(c_double), value :: rmin, rmax
      integer(c_int32_t), value :: nbins, nmu, logbins
    end function
    integer(c_int) function gr_count_2pcf(ctx, N2, N3, counts, catsum) &
        bind(c, name="gr_count_2pcf")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), catsum(*)
      integer(c_int64_t) :: counts(*)
    end function
    integer(c_int) function gr_count_3pcf(ctx, N2, N3, counts, catsum) &
        bind(c, name="gr_count_3pcf")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), catsum(*)
      integer(c_int64_t) :: counts(*)
    end function
    integer(c_int) function gr_count_4pcf(ctx, N2, N3, discN, discR, counts, catsum, &
        dcount, dsum) bind(c, name="gr_count_4pcf")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), discN(*), discR(*), catsum(*), dsum(*)
      integer(c_int64_t) :: counts(*), dcount(*)
    end function
    integer(c_int) function gr_set_regions(ctx, nsplit) bind(c, name="gr_set_regions")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsplit
    end function
    integer(c_int) function gr_count_2pcf_batched(ctx, N2, N3, counts, catsum) &
        bind(c, name="gr_count_2pcf_batched")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), catsum(*)
      integer(c_int64_t) :: counts(*)
    end function
    integer(c_int) function gr_set_region_ids(ctx, region_of_point, nregions) &
        bind(c, name="gr_set_region_ids")
      import :: c_ptr, c_int, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: region_of_point(*)   ! 0-based region of every point
      integer(c_int32_t), value :: nregions
    end function
    integer(c_int) function gr_set_mocks(ctx, nmocks, n_data, n_rand) bind(c, name="gr_set_mocks")
      import :: c_ptr, c_int, c_int32_t, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nmocks
      integer(c_int64_t), intent(in) :: n_data(*), n_rand(*)
    end function
    integer(c_int) function gr_count_2pcf_regions(ctx, N2, N3, counts, catsum) &
        bind(c, name="gr_count_2pcf_regions")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), catsum(*)   ! (nbins, nmu, nregions) ...
      integer(c_int64_t) :: counts(*)
    end function
    integer(c_int) function gr_count_3pcf_batched(ctx, N2, N3, counts, catsum) &
        bind(c, name="gr_count_3pcf_batched")
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: N2(*), N3(*), catsum(*)
      integer(c_int64_t) :: counts(*)
    end function
  end interface
end module gramsci_cuda
