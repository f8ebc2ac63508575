      !> @file
      !> iso_c_binding interface of the B200 DIM time-step library
      !> (libdim2d.so, C declarations in include/dim2d.h) for the
      !> reference's Fortran host.
      !
      !> @brief
      !> Fortran views of the C entry points that the GPU time
      !> integrator (td_integrator_class.f beside this file) calls:
      !> one bind(C) interface per function, the bind(C) copy of the
      !> dim2d_params struct, and dim2d_check, which turns a non-zero
      !> status into the reference's way of failing (a message and
      !> `stop`, src/parameters/errors_module.f).
      !
      !> Argument passing follows include/dim2d.h: scalars by value,
      !> arrays and structs by reference, the handle as type(c_ptr).
      !> nodes(nx,ny,ne) is passed as is: its Fortran column-major
      !> layout is the library's input layout.
      !-----------------------------------------------------------------
      module dim2d_gpu_interface

        use iso_c_binding, only :
     $       c_int,
     $       c_double,
     $       c_ptr,
     $       c_char,
     $       c_null_char,
     $       c_associated,
     $       c_f_pointer

        implicit none

        private
        public ::
     $       dim2d_params_t,
     $       DIM2D_FP64,
     $       DIM2D_MIXED,
     $       dim2d_default_params,
     $       dim2d_create,
     $       dim2d_upload,
     $       dim2d_step,
     $       dim2d_download,
     $       dim2d_time_dev,
     $       dim2d_apply_bc_on_nodes,
     $       dim2d_sync,
     $       dim2d_destroy,
     $       dim2d_check


        !> precision of the stencil / flux pass (include/dim2d.h)
        integer(c_int), parameter :: DIM2D_FP64  = 0
        integer(c_int), parameter :: DIM2D_MIXED = 1


        !> @brief C struct dim2d_params (include/dim2d.h): the
        !> physical and boundary constants the reference keeps as
        !> compile-time parameters (dim2d_parameters.f,
        !> parameters_input.f)
        !---------------------------------------------------------------
        type, bind(C) :: dim2d_params_t
          real(c_double) :: re
          real(c_double) :: we
          real(c_double) :: pr
          real(c_double) :: cv_r
          real(c_double) :: viscous_r
          integer(c_int) :: gravity_ac
          real(c_double) :: gravity
          real(c_double) :: wall_micro_contact_angle
          integer(c_int) :: wall_heat_source_choice
          real(c_double) :: wall_maximum_heat_flux
          real(c_double) :: wall_heat_source_center
          real(c_double) :: wall_heat_source_variance
          integer(c_int) :: obc_eigenqties_strategy
          integer(c_int) :: obc_edge_flux_strategy
          real(c_double) :: T0
          real(c_double) :: flow_velocity
        end type dim2d_params_t


        interface

          subroutine dim2d_default_params(p)
     $         bind(C, name='dim2d_default_params')
            import dim2d_params_t
            type(dim2d_params_t), intent(out) :: p
          end subroutine dim2d_default_params

          function dim2d_create(p, nx, ny, bc_choice, bc_type,
     $         bc_order, precision, h)
     $         bind(C, name='dim2d_create')
            import dim2d_params_t, c_int, c_ptr
            type(dim2d_params_t)        , intent(in)  :: p
            integer(c_int), value                     :: nx
            integer(c_int), value                     :: ny
            integer(c_int), dimension(8), intent(in)  :: bc_choice
            integer(c_int), dimension(8), intent(in)  :: bc_type
            integer(c_int), dimension(8), intent(in)  :: bc_order
            integer(c_int), value                     :: precision
            type(c_ptr)                 , intent(out) :: h
            integer(c_int)                            :: dim2d_create
          end function dim2d_create

          function dim2d_upload(h, nodes, x_map, y_map, t)
     $         bind(C, name='dim2d_upload')
            import c_int, c_double, c_ptr
            type(c_ptr)   , value                   :: h
            real(c_double), dimension(*), intent(in) :: nodes
            real(c_double), dimension(*), intent(in) :: x_map
            real(c_double), dimension(*), intent(in) :: y_map
            real(c_double), value                   :: t
            integer(c_int)                          :: dim2d_upload
          end function dim2d_upload

          function dim2d_step(h, dt, nsteps)
     $         bind(C, name='dim2d_step')
            import c_int, c_double, c_ptr
            type(c_ptr)   , value :: h
            real(c_double), value :: dt
            integer(c_int), value :: nsteps
            integer(c_int)        :: dim2d_step
          end function dim2d_step

          function dim2d_download(h, nodes, t)
     $         bind(C, name='dim2d_download')
            import c_int, c_double, c_ptr
            type(c_ptr)   , value                      :: h
            real(c_double), dimension(*), intent(inout) :: nodes
            real(c_double)              , intent(out)   :: t
            integer(c_int)                             :: dim2d_download
          end function dim2d_download

          function dim2d_time_dev(h, time_dev)
     $         bind(C, name='dim2d_time_dev')
            import c_int, c_double, c_ptr
            type(c_ptr)   , value                      :: h
            real(c_double), dimension(*), intent(inout) :: time_dev
            integer(c_int)                             :: dim2d_time_dev
          end function dim2d_time_dev

          function dim2d_apply_bc_on_nodes(h)
     $         bind(C, name='dim2d_apply_bc_on_nodes')
            import c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int)     :: dim2d_apply_bc_on_nodes
          end function dim2d_apply_bc_on_nodes

          function dim2d_sync(h) bind(C, name='dim2d_sync')
            import c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int)     :: dim2d_sync
          end function dim2d_sync

          function dim2d_destroy(h) bind(C, name='dim2d_destroy')
            import c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int)     :: dim2d_destroy
          end function dim2d_destroy

          function dim2d_last_error()
     $         bind(C, name='dim2d_last_error')
            import c_ptr
            type(c_ptr) :: dim2d_last_error
          end function dim2d_last_error

        end interface


        contains


        !> @brief stop with the library's message when a call
        !> returned a non-zero status (the reference stops on errors,
        !> src/parameters/errors_module.f)
        !
        !> @param rc
        !> status returned by the call
        !
        !> @param where
        !> name of the call, for the message
        !--------------------------------------------------------------
        subroutine dim2d_check(rc, where)

          implicit none

          integer(c_int), intent(in) :: rc
          character(*)  , intent(in) :: where

          type(c_ptr)                                  :: msg_ptr
          character(kind=c_char), dimension(:), pointer :: msg
          character(len=1024)                          :: text
          integer                                      :: i, n

          if(rc.eq.0) return

          msg_ptr = dim2d_last_error()
          n    = 0
          text = ' '
          if(c_associated(msg_ptr)) then
             call c_f_pointer(msg_ptr, msg, [1024])
             do i=1,1024
                if(msg(i).eq.c_null_char) exit
                text(i:i) = msg(i)
                n = i
             end do
          end if
          write(*,'(3A,I0,2A)')
     $         'dim2d_gpu_interface: ', where, ' failed (', rc, '): ',
     $         text(1:max(n,1))
          stop 'dim2d_gpu_interface: library call failed'

        end subroutine dim2d_check

      end module dim2d_gpu_interface
