! module_pepcg.f90 -- iso_c_binding interface to libpepcg (include/pepcg.h) and
! drop-in bodies for the two library routines that PEPC frontends call through
! module_pepc (pepc_grow_tree, pepc_traverse_tree; src/treecode/lpepcsrc/module_pepc.f90:435-468).
!
! A PEPC build that links libpepcg replaces the bodies of libpepc_grow_tree
! and libpepc_traverse_tree (module_libpepc_main.f90:105-124, :161-200) with
! calls to pepcg_grow_and_sort / pepcg_traverse below; everything the frontends
! see (t_particle arrays, key order after grow, accumulated results) stays as
! in the reference.  Compiles with any Fortran 2003 compiler that has
! iso_c_binding; link with -lpepcg -lcudart -lstdc++.
module module_pepcg
   use, intrinsic :: iso_c_binding
   implicit none
   private

   integer(c_int), parameter, public :: PEPCG_OK = 0
   integer(c_int), parameter, public :: PEPCG_WARN_NOT_NEUTRAL = 100
   integer(c_int32_t), parameter, public :: PEPCG_PRECISION_PLAIN = 0, PEPCG_PRECISION_MIXED = 1
   integer(c_int32_t), parameter, public :: PEPCG_WALK_PER_TARGET = 0, PEPCG_WALK_PER_TILE = 1, &
                                            PEPCG_WALK_GROUP = 2

   type, bind(c), public :: pepcg_params
      real(c_double) :: theta2, eps2
      integer(c_int32_t) :: force_law, mac_select, curve, precision, walk, tile_size
      integer(c_int32_t) :: force_cubic_domain
      integer(c_int32_t) :: periodicity(3)
      integer(c_int32_t) :: mirror_box_layers, include_far_field_if_periodic
      integer(c_int32_t) :: fmm_extrinsic_correction
      real(c_double) :: t_lattice_1(3), t_lattice_2(3), t_lattice_3(3), lattice_origin(3)
      integer(c_int32_t) :: device
      integer(c_int32_t) :: overwrite_results
      real(c_double) :: kelbg_invsqrttemp
      integer(c_int32_t) :: group_size
      integer(c_int32_t) :: reserved0
      real(c_double) :: spatial_interaction_cutoff(3)
      integer(c_int32_t) :: reserved(4)
   end type

   interface
      subroutine pepcg_params_default(p) bind(c, name="pepcg_params_default")
         import :: pepcg_params
         type(pepcg_params), intent(out) :: p
      end subroutine
      integer(c_int) function pepcg_create(ctx, p) bind(c, name="pepcg_create")
         import :: c_int, c_ptr, pepcg_params
         type(c_ptr), intent(out) :: ctx
         type(pepcg_params), intent(in) :: p
      end function
      integer(c_int) function pepcg_destroy(ctx) bind(c, name="pepcg_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      type(c_ptr) function pepcg_last_error(ctx) bind(c, name="pepcg_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pepcg_grow_tree(ctx, n, x, y, z, q, key_out, perm_out, &
                                              x_out, y_out, z_out) bind(c, name="pepcg_grow_tree")
         import :: c_int, c_ptr, c_int64_t, c_double
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: n
         real(c_double), intent(in) :: x(*), y(*), z(*), q(*)
         integer(c_int64_t), intent(out) :: key_out(*), perm_out(*)
         real(c_double), intent(out) :: x_out(*), y_out(*), z_out(*)
      end function
      integer(c_int) function pepcg_traverse_tree(ctx, nt, tx, ty, tz, tkeys, ex, ey, ez, &
                                                  pot, work) bind(c, name="pepcg_traverse_tree")
         import :: c_int, c_ptr, c_int64_t, c_double
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: nt
         real(c_double), intent(in) :: tx(*), ty(*), tz(*)
         integer(c_int64_t), intent(in) :: tkeys(*)
         real(c_double), intent(inout) :: ex(*), ey(*), ez(*), pot(*), work(*)
      end function
      integer(c_int) function pepcg_timber_tree(ctx) bind(c, name="pepcg_timber_tree")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pepcg_sort_keys(ctx, n, keys, keys_out, perm_out) &
         bind(c, name="pepcg_sort_keys")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: n
         integer(c_int64_t), intent(in) :: keys(*)
         integer(c_int64_t), intent(out) :: keys_out(*), perm_out(*)
      end function
      integer(c_int) function pepcg_lattice_force(ctx, pos, e, phi) &
         bind(c, name="pepcg_lattice_force")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: pos(3)
         real(c_double), intent(out) :: e(3), phi
      end function
   end interface

   public :: pepcg_params_default, pepcg_create, pepcg_destroy, pepcg_last_error
   public :: pepcg_grow_tree, pepcg_traverse_tree, pepcg_timber_tree
   public :: pepcg_sort_keys, pepcg_lattice_force
   public :: pepcg_init_from_namelists, pepcg_grow_and_sort, pepcg_traverse

   type(c_ptr), save, public :: pepcg_ctx = c_null_ptr

contains

   !> fills the parameters from the reference's namelist variables
   !> (/calc_force_coulomb/ theta2, eps2; /libpepc/ periodicity, mirror_box_layers,
   !> force_cubic_domain; the frontend's spatial_interaction_cutoff, e.g. pepc-mini's
   !> /pepcmini/ namelist, frontends/pepc-mini/module_helper.f90:82-90) and creates the
   !> context
   subroutine pepcg_init_from_namelists(theta2, eps2, periodicity, mirror_box_layers, &
                                        force_cubic_domain, walk, precision, &
                                        spatial_interaction_cutoff)
      real(c_double), intent(in) :: theta2, eps2
      logical, intent(in) :: periodicity(3), force_cubic_domain
      integer, intent(in) :: mirror_box_layers
      integer(c_int32_t), intent(in) :: walk, precision
      real(c_double), intent(in) :: spatial_interaction_cutoff(3)
      type(pepcg_params) :: p
      integer(c_int) :: rc
      integer :: d
      call pepcg_params_default(p)
      p%theta2 = theta2
      p%eps2 = eps2
      do d = 1, 3
         p%periodicity(d) = merge(1_c_int32_t, 0_c_int32_t, periodicity(d))
      end do
      p%mirror_box_layers = int(mirror_box_layers, c_int32_t)
      p%force_cubic_domain = merge(1_c_int32_t, 0_c_int32_t, force_cubic_domain)
      p%walk = walk
      p%precision = precision
      p%spatial_interaction_cutoff = spatial_interaction_cutoff
      rc = pepcg_create(pepcg_ctx, p)
      if (rc /= PEPCG_OK) stop "pepcg_create failed"
   end subroutine

   !> body of libpepc_grow_tree: x, q in; particles reordered into key order,
   !> key set, coordinates rewritten where a duplicate key was shifted,
   !> work = 1 and node_leaf = -1 (module_domains.f90:316-318)
   subroutine pepcg_grow_and_sort(n, x, q, key, work, perm)
      integer(c_int64_t), intent(in) :: n
      real(c_double), intent(inout) :: x(:, :)        ! (3, n), reordered on return
      real(c_double), intent(inout) :: q(:)           ! reordered on return
      integer(c_int64_t), intent(out) :: key(:)
      real(c_double), intent(out) :: work(:)
      integer(c_int64_t), intent(out) :: perm(:)      ! 0-based source index of each result
      real(c_double), allocatable :: xs(:), ys(:), zs(:), xo(:), yo(:), zo(:), qo(:)
      integer(c_int) :: rc
      allocate (xs(n), ys(n), zs(n), xo(n), yo(n), zo(n), qo(n))
      xs = x(1, 1:n); ys = x(2, 1:n); zs = x(3, 1:n)
      rc = pepcg_grow_tree(pepcg_ctx, n, xs, ys, zs, q, key, perm, xo, yo, zo)
      if (rc /= PEPCG_OK .and. rc /= PEPCG_WARN_NOT_NEUTRAL) stop "pepcg_grow_tree failed"
      qo = q(perm(1:n) + 1)
      x(1, 1:n) = xo; x(2, 1:n) = yo; x(3, 1:n) = zo
      q(1:n) = qo
      work(1:n) = 1.0_c_double
   end subroutine

   !> body of libpepc_traverse_tree: accumulates e, pot and work like
   !> calc_force_per_interaction_* (+= onto particle%results)
   subroutine pepcg_traverse(nt, x, key, e, pot, work)
      integer(c_int64_t), intent(in) :: nt
      real(c_double), intent(in) :: x(:, :)
      integer(c_int64_t), intent(in) :: key(:)
      real(c_double), intent(inout) :: e(:, :), pot(:), work(:)
      real(c_double), allocatable :: tx(:), ty(:), tz(:), ex(:), ey(:), ez(:)
      integer(c_int) :: rc
      allocate (tx(nt), ty(nt), tz(nt), ex(nt), ey(nt), ez(nt))
      tx = x(1, 1:nt); ty = x(2, 1:nt); tz = x(3, 1:nt)
      ex = e(1, 1:nt); ey = e(2, 1:nt); ez = e(3, 1:nt)
      rc = pepcg_traverse_tree(pepcg_ctx, nt, tx, ty, tz, key, ex, ey, ez, pot, work)
      if (rc /= PEPCG_OK .and. rc /= PEPCG_WARN_NOT_NEUTRAL) stop "pepcg_traverse_tree failed"
      e(1, 1:nt) = ex; e(2, 1:nt) = ey; e(3, 1:nt) = ez
   end subroutine
end module module_pepcg
