      !> @file
      !> RK3-TVD time integrator of one DIM field on a B200 GPU: the
      !> drop-in replacement of
      !> src/td_integrator/rungekutta3rdtvd/td_integrator_class.f
      !
      !> @brief
      !> Same module name, type name and type-bound procedures as the
      !> reference's integrator (td_integrator_abstract_class.f:39-77),
      !> so field_class.f compiles against it unchanged; the build
      !> selects this directory instead of rungekutta3rdtvd/.
      !> integrate(field_used, dt) advances field_used%nodes by one
      !> RK3 step (td_integrator_class.f:103-161 of the reference:
      !> three stages, each with compute_time_dev, the stage update and
      !> apply_bc_on_nodes) through the C library (include/dim2d.h).
      !
      !> The field stays in GPU memory between calls.  The first call
      !> creates the library's handle from the run's compile-time
      !> parameters (parameters_input.f, dim2d_parameters.f) and
      !> uploads nodes, x_map, y_map and time.  field_used%nodes on the
      !> host is brought up to date after exactly the steps at which
      !> the reference's driver reads it (src/main/sim_dim2d.f:55-92):
      !> the output steps of detail_print, the end of the time loop
      !> (steady-state check, final output).  A program that reads or
      !> changes field_used%nodes at other steps calls
      !> dim2d_gpu_sync_field (device -> host) or
      !> dim2d_gpu_upload_field (host -> device) around that access,
      !> or sets gpu_sync_every_step = .true.
      !
      !> One field per process, as the reference's drivers use it.
      !> integrate_ext (the buffer-layer domain extension) is not
      !> provided on the GPU: it stops with a message.
      !-----------------------------------------------------------------
      module td_integrator_class

        use iso_c_binding, only :
     $       c_int,
     $       c_double,
     $       c_ptr,
     $       c_null_ptr,
     $       c_associated

        use dim2d_gpu_interface, only :
     $       dim2d_params_t,
     $       DIM2D_FP64,
     $       dim2d_default_params,
     $       dim2d_create,
     $       dim2d_upload,
     $       dim2d_step,
     $       dim2d_download,
     $       dim2d_destroy,
     $       dim2d_check

        use dim2d_parameters, only :
     $       re,
     $       we,
     $       pr,
     $       cv_r,
     $       viscous_r,
     $       gravity

        use field_abstract_class, only :
     $       field_abstract

        use parameters_input, only :
     $       nx,ny,ne,
     $       t_max,
     $       dt_run => dt,
     $       detail_print,
     $       steady_state_simulation,
     $       T0,
     $       flow_velocity,
     $       gravity_ac,
     $       bc_N_choice, bc_S_choice, bc_E_choice, bc_W_choice,
     $       bc_NE_choice, bc_NW_choice, bc_SE_choice, bc_SW_choice,
     $       bc_N_type_choice, bc_S_type_choice,
     $       bc_E_type_choice, bc_W_type_choice,
     $       bc_NE_type_choice, bc_NW_type_choice,
     $       bc_SE_type_choice, bc_SW_type_choice,
     $       bc_order1, bc_order2, bc_order3, bc_order4,
     $       bc_order5, bc_order6, bc_order7, bc_order8,
     $       wall_micro_contact_angle,
     $       wall_heat_source_choice,
     $       wall_maximum_heat_flux,
     $       wall_heat_source_center,
     $       wall_heat_source_variance,
     $       obc_eigenqties_strategy,
     $       obc_edge_flux_strategy

        use parameters_kind, only :
     $       rkind,
     $       ikind

        use td_integrator_abstract_class, only :
     $       td_integrator_abstract

        implicit none


        private
        public ::
     $       td_integrator,
     $       dim2d_gpu_sync_field,
     $       dim2d_gpu_upload_field,
     $       dim2d_gpu_release,
     $       gpu_precision,
     $       gpu_sync_every_step


        !> @class td_integrator
        !> RK3-TVD integration of the field on the GPU
        !---------------------------------------------------------------
        type, extends(td_integrator_abstract) :: td_integrator

          contains

          procedure, nopass :: integrate
          procedure, nopass :: integrate_ext

        end type td_integrator


        !> precision of the stencil / flux pass: DIM2D_FP64 (the
        !> reference's arithmetic) or DIM2D_MIXED; set before the
        !> first integrate
        integer(c_int), save :: gpu_precision = DIM2D_FP64

        !> bring field_used%nodes up to date after every step
        logical, save :: gpu_sync_every_step = .false.

        ! handle of the field's solver and the step count since the
        ! upload (the driver's loop counter t + s*nt)
        type(c_ptr)   , save :: handle = c_null_ptr
        integer(ikind), save :: steps_done = 0
        integer(ikind), save :: nt_loop = 0
        integer(ikind), save :: output_print = 0


        contains


        !> @brief one RK3-TVD step of the field on the GPU
        !
        !> @param field_used
        !> object encapsulating the main variables
        !
        !> @param dt
        !> time step integrated
        !--------------------------------------------------------------
        subroutine integrate(field_used, dt)

          implicit none

          class(field_abstract), intent(inout) :: field_used
          real(rkind)          , intent(in)    :: dt

          if(.not.c_associated(handle)) then
             call dim2d_gpu_upload_field(field_used)
          end if

          call dim2d_check(
     $         dim2d_step(handle, real(dt,c_double), 1_c_int),
     $         'dim2d_step')
          steps_done = steps_done + 1

          if(host_reads_nodes()) then
             call dim2d_gpu_sync_field(field_used)
          end if

        end subroutine integrate


        !> @brief integration of the domain and its buffer layers:
        !> not provided on the GPU (the buffer-layer extension stays
        !> with the reference's host code)
        !
        !> @param field_used
        !> object encapsulating the main variables
        !
        !> @param dt
        !> time step integrated
        !--------------------------------------------------------------
        subroutine integrate_ext(field_used, dt)

          implicit none

          class(field_abstract), intent(inout) :: field_used
          real(rkind)          , intent(in)    :: dt

          write(*,'(A,ES12.5,A,ES12.5)')
     $         'td_integrator (GPU): integrate_ext called at t=',
     $         field_used%time, ', dt=', dt
          stop 'td_integrator (GPU): integrate_ext not provided'

        end subroutine integrate_ext


        !> @brief create the solver on first use and copy the field's
        !> nodes, x_map, y_map and time to the GPU; restarts the output
        !> schedule from this state
        !
        !> @param field_used
        !> object encapsulating the main variables
        !--------------------------------------------------------------
        subroutine dim2d_gpu_upload_field(field_used)

          implicit none

          class(field_abstract), intent(inout) :: field_used

          type(dim2d_params_t)         :: p
          integer(c_int), dimension(8) :: bc_choice
          integer(c_int), dimension(8) :: bc_type
          integer(c_int), dimension(8) :: bc_order

          if(.not.c_associated(handle)) then

             ! dim2d_parameters.f:146-199, parameters_input.f:127-662
             call dim2d_default_params(p)
             p%re        = re
             p%we        = we
             p%pr        = pr
             p%cv_r      = cv_r
             p%viscous_r = viscous_r
             p%gravity_ac = 0
             if(gravity_ac) p%gravity_ac = 1
             p%gravity                   = gravity
             p%wall_micro_contact_angle  = wall_micro_contact_angle
             p%wall_heat_source_choice   = wall_heat_source_choice
             p%wall_maximum_heat_flux    = wall_maximum_heat_flux
             p%wall_heat_source_center   = wall_heat_source_center
             p%wall_heat_source_variance = wall_heat_source_variance
             p%obc_eigenqties_strategy   = obc_eigenqties_strategy
             p%obc_edge_flux_strategy    = obc_edge_flux_strategy
             p%T0            = T0
             p%flow_velocity = flow_velocity

             ! sections in the library's slot order N,S,E,W,NE,NW,SE,SW
             ! (the same numbers as parameters_constant.f:145-172)
             bc_choice = [bc_N_choice, bc_S_choice, bc_E_choice,
     $            bc_W_choice, bc_NE_choice, bc_NW_choice,
     $            bc_SE_choice, bc_SW_choice]
             bc_type = [bc_N_type_choice, bc_S_type_choice,
     $            bc_E_type_choice, bc_W_type_choice,
     $            bc_NE_type_choice, bc_NW_type_choice,
     $            bc_SE_type_choice, bc_SW_type_choice]
             bc_order = [bc_order1, bc_order2, bc_order3, bc_order4,
     $            bc_order5, bc_order6, bc_order7, bc_order8]

             call dim2d_check(
     $            dim2d_create(p, int(nx,c_int), int(ny,c_int),
     $            bc_choice, bc_type, bc_order, gpu_precision,
     $            handle),
     $            'dim2d_create')

          end if

          if(ne.ne.4) then
             stop 'td_integrator (GPU): the DIM field has ne=4'
          end if

          call dim2d_check(
     $         dim2d_upload(handle, field_used%nodes, field_used%x_map,
     $         field_used%y_map, real(field_used%time,c_double)),
     $         'dim2d_upload')

          ! the driver's time loop from this state (sim_dim2d.f:55-60)
          steps_done = 0
          if(steady_state_simulation) then
             nt_loop = int(t_max/dt_run)
          else
             nt_loop = int((t_max-field_used%time)/dt_run)
          end if
          if(detail_print.gt.0.0d0) then
             output_print = int(1.0d0/detail_print)
          else
             output_print = 0
          end if

        end subroutine dim2d_gpu_upload_field


        !> @brief copy the GPU state into field_used%nodes
        !
        !> @param field_used
        !> object encapsulating the main variables
        !--------------------------------------------------------------
        subroutine dim2d_gpu_sync_field(field_used)

          implicit none

          class(field_abstract), intent(inout) :: field_used

          real(c_double) :: t_device

          if(.not.c_associated(handle)) return
          call dim2d_check(
     $         dim2d_download(handle, field_used%nodes, t_device),
     $         'dim2d_download')

        end subroutine dim2d_gpu_sync_field


        !> @brief free the GPU solver (its memory and streams)
        !--------------------------------------------------------------
        subroutine dim2d_gpu_release()

          implicit none

          if(c_associated(handle)) then
             call dim2d_check(dim2d_destroy(handle), 'dim2d_destroy')
             handle = c_null_ptr
          end if

        end subroutine dim2d_gpu_release


        !> @brief whether the reference's driver reads field%nodes
        !> after the step just taken: an output step
        !> (sim_dim2d.f:86-89) or the end of a pass of the time loop
        !> (steady-state check and final output, sim_dim2d.f:93-111)
        !--------------------------------------------------------------
        function host_reads_nodes()

          implicit none

          logical :: host_reads_nodes

          host_reads_nodes = gpu_sync_every_step
          if(output_print.eq.1) then
             host_reads_nodes = .true.
          else if(output_print.ne.0) then
             if(mod(steps_done,output_print).eq.0) then
                host_reads_nodes = .true.
             end if
          end if
          if(nt_loop.gt.0) then
             if(mod(steps_done,nt_loop).eq.0) then
                host_reads_nodes = .true.
             end if
          end if

        end function host_reads_nodes

      end module td_integrator_class
